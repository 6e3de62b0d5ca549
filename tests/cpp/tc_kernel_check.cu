// GPU check of the tensor-core update (k_tc_pack + k_trail_tc) against an
// FP64 CPU reference: fronts of assorted sizes (odd n and N, fronts without
// an update), outer panels (w = 512) and sub-panels with a column bound
// (w = 128), three-term and plain TF32 and plain BF16.  Every entry the update
// must change is compared with C - P P^T computed in double (relative to the
// sum of the products' magnitudes: 1e-5 for three terms, 2e-3 for plain TF32,
// 1.6e-2 for BF16, whose operands keep 8 bits); every
// other entry of every front must be untouched, and the error word clear.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../updating-multifrontal_b200/csrc/kernels_tc.cu"
namespace mfgpu { std::atomic<long long> g_launches{0}; }
using namespace mfgpu;
#define CK(x) do { cudaError_t ce_ = (x); if (ce_ != cudaSuccess) { printf("CUDA %s at %d: %s\n", #x, __LINE__, cudaGetErrorString(ce_)); return 1; } } while (0)

int run(int K, int split, std::vector<int> n, std::vector<int> N, int w = 512, int cend = -1) {
  const int nf = n.size();
  std::vector<FrontDev> fr(nf);
  int64_t off = 0;
  for (int i = 0; i < nf; i++) {
    fr[i] = FrontDev{};
    fr[i].off = off; fr[i].dof_off = 0; fr[i].n = n[i]; fr[i].m = N[i] - n[i]; fr[i].N = N[i];
    fr[i].ld = (N[i] + 7) & ~7; off += ((int64_t)fr[i].ld * N[i] + 31) / 32 * 32;
  }
  std::vector<float> h(off);
  srand(12345);
  for (auto& v : h) v = (float)rand() / RAND_MAX * 2.0f - 1.0f;
  float* dF; int* dl; FrontDev* dfr; DevError* derr;
  CK(cudaMalloc(&dF, off * 4)); CK(cudaMalloc(&dl, nf * 4)); CK(cudaMalloc(&dfr, nf * sizeof(FrontDev)));
  CK(cudaMalloc(&derr, sizeof(DevError)));
  CK(cudaMemset(derr, 0, sizeof(DevError)));
  std::vector<int> ids(nf); for (int i = 0; i < nf; i++) ids[i] = i;
  CK(cudaMemcpy(dF, h.data(), off * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dl, ids.data(), nf * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dfr, fr.data(), nf * sizeof(FrontDev), cudaMemcpyHostToDevice));
  const int64_t nt = tc_tiles(n, N, K, w, cend);
  const int cap = tc_pack_cap(n, N, K, w);
  void* dpack = nullptr;
  CK(cudaMalloc(&dpack, std::max<size_t>(16, tc_pack_bytes(nf, cap))));
  CK(launch_tc_pack(dl, nf, cap, dfr, dF, K, w, split, dpack, 0));
  CK(launch_trail_tc(dl, nf, nt, dfr, dF, K, w, cend, split, cap, dpack, derr, 0));
  CK(cudaDeviceSynchronize());
  DevError e; CK(cudaMemcpy(&e, derr, sizeof e, cudaMemcpyDeviceToHost));
  std::vector<float> g(off);
  CK(cudaMemcpy(g.data(), dF, off * 4, cudaMemcpyDeviceToHost));
  double maxerr = 0; long long bad_untouched = 0, checked = 0, nbad = 0;
  for (int i = 0; i < nf; i++) {
    const FrontDev& d = fr[i];
    const float* A = h.data() + d.off; const float* G = g.data() + d.off;
    const int k1 = std::min(K + w, d.n);
    const int cmax = cend < 0 ? d.N : std::min(cend, d.n);
    for (int c = 0; c < d.N; c++)
      for (int r = 0; r < d.ld; r++) {
        const int64_t idx = r + (int64_t)c * d.ld;
        const bool upd = K < d.n && c >= k1 && c < cmax && r >= c && r < d.N;
        if (!upd) { if (G[idx] != A[idx]) bad_untouched++; continue; }
        double s = 0, sa = 0;
        for (int k = K; k < k1; k++) { double p = (double)A[r + (int64_t)k * d.ld] * A[c + (int64_t)k * d.ld]; s += p; sa += fabs(p); }
        const double ref = (double)A[idx] - s;
        const double e_ = fabs(G[idx] - ref) / std::max(1.0, sa);
        maxerr = std::max(maxerr, e_);
        if (e_ > 1e-3) { nbad++; if (nbad <= 8) printf("  bad f%d r=%d c=%d G=%.5f ref=%.5f A=%.5f\n", i, r, c, G[idx], ref, A[idx]); }
        checked++;
      }
  }
  printf("w=%d cend=%d K=%d split=%d tiles=%lld err=%d checked=%lld max_rel_err=%.3e untouched_bad=%lld nbad=%lld\n", w, cend, K,
         split, (long long)nt, e.code, checked, maxerr, bad_untouched, nbad);
  cudaFree(dF); cudaFree(dl); cudaFree(dfr); cudaFree(derr); cudaFree(dpack);
  return (e.code != 0 || bad_untouched ||
          maxerr > (split == 3 ? 1e-5 : split == 1 ? 2e-3 : 1.6e-2)) ? 2 : 0;
}

int main() {
  int rc = 0;
  for (int split : {3, 1, 2}) {
    rc |= run(0, split, {600, 300, 1000}, {1000, 300, 1300});
    rc |= run(256, split, {600, 300, 1000}, {1000, 300, 1300});
    rc |= run(512, split, {600, 300, 1000}, {1000, 300, 1300});
    rc |= run(0, split, {100}, {129});
    rc |= run(0, split, {601, 99, 1001, 7}, {1003, 131, 1001, 141});
    rc |= run(512, split, {1001, 515}, {1601, 1283});
    rc |= run(0, split, {600, 300, 1000}, {1000, 300, 1300}, 128, 512);
    rc |= run(128, split, {601, 99, 1001, 7}, {1003, 131, 1001, 141}, 128, 512);
    rc |= run(384, split, {1001, 515, 1024}, {1601, 1283, 2000}, 128, 512);
    rc |= run(640, split, {1001, 515, 1024}, {1601, 1283, 2000}, 128, 1024);
    rc |= run(0, split, {2000}, {2300}, 128, 512);
  }
  printf(rc ? "FAILED\n" : "ok\n");
  return rc;
}
