// Panel-by-panel partial Cholesky without grid barriers (both precisions).
//
// The reference factors a front's pivot block and forms its Schur complement
// in one dense LU call sequence (src/DE/mf2d.cpp:558-576).  Here, for the
// fronts of one tree level, every W-column panel [Ks, Ks + kb) (kb = min(W,
// n - Ks)) takes two launches:
//   k_subpanel     every CTA loads the kb x kb diagonal block into shared memory
//                  and factors it itself (right-looking Cholesky; the same
//                  arithmetic in every CTA), then takes 128-row blocks of the
//                  rows below, solves them against it (X <- X L^{-T}, each
//                  row by two threads) and writes them back; the first item
//                  of a front leaves the factored block in a scratch slot
//                  (the front's own copy is still being read by other CTAs),
//                  and k_panel_diag, the next launch, puts it in place;
//   k_trail_syrk   the trailing lower triangle, C(k1:N, k1:N) -= P P^T with
//                  P = L(k1:N, Ks:k1), in 64 x 64 tiles (FP64: DMMA m8n8k4;
//                  FP32: FFMA), all fronts' tiles over all SMs.
// Every element of a panel is read and written once by k_subpanel and no CTA
// waits for another, so a level of a few small fronts (the top of a 2D tree)
// costs two short launches per panel instead of two grid barriers per 32
// columns.  The tensor-core levels of the mixed path use k_subpanel alone for
// their 128-column sub-panels (their updates run on the tensor cores).
// A non-positive pivot records error code 1.
#include <algorithm>
#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int kSubRows = 128;             // rows per solve item
constexpr int kSubThreads = 256;

template <class T>
__device__ __forceinline__ T rsq(T x);
template <>
__device__ __forceinline__ float rsq<float>(float x) { return rsqrtf(x); }
template <>
__device__ __forceinline__ double rsq<double>(double x) { return rsqrt(x); }

template <int W>
constexpr int sub_stride() { return W + 1; }

template <class T, int W>
constexpr size_t sub_smem() {
  return ((size_t)(W + kSubRows) * sub_stride<W>() + (size_t)(W / 32) * 32 * 33) * sizeof(T);
}

// One warp factors the 32 x 32 (jb x jb) diagonal block at (j0, j0) of Ds in
// place (lane i holds row i in registers; Cholesky by shuffles) and writes the
// inverse of the factor to Li (row-major, stride 33).  Returns the first
// non-positive pivot column of the block or -1.
template <class T, int S>
__device__ int warp_chol_inv(T* Ds, int j0, int jb, T* Li) {
  const int lane = threadIdx.x & 31;
  T row[32];
#pragma unroll
  for (int t = 0; t < 32; t++)
    row[t] = (lane < jb && t <= lane) ? Ds[(j0 + lane) * S + j0 + t] : T(0);
  int bad = -1;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    if (j < jb) {
      T djj = __shfl_sync(0xffffffffu, row[j], j);
      if (!(djj > T(0))) {                 // non-positive or NaN pivot: not SPD
        if (bad < 0) bad = j;
        djj = T(1);
      }
      const T r = rsq<T>(djj);
      if (lane == j) row[j] = djj * r;
      else if (lane > j) row[j] = row[j] * r;
#pragma unroll
      for (int l = j + 1; l < 32; l++) {
        const T llj = __shfl_sync(0xffffffffu, row[j], l);
        if (lane >= l && l < jb) row[l] -= row[j] * llj;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 32; t++)
    if (lane < jb && t <= lane) Ds[(j0 + lane) * S + j0 + t] = row[t];
  __syncwarp();
  // lane c: column c of the inverse, x_i = (delta_ic - sum_{c<=t<i} L(i,t) x_t) / L(i,i)
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) {
    T v = T(0);
    if (i < jb && i >= lane) {
      T acc = i == lane ? T(1) : T(0);
#pragma unroll
      for (int t = 0; t < i; t++)
        if (t >= lane) acc -= Ds[(j0 + i) * S + j0 + t] * x[t];
      v = acc / Ds[(j0 + i) * S + j0 + i];
    }
    x[i] = v;
    Li[i * 33 + lane] = v;
  }
  __syncwarp();
  return bad;
}

// Row `r` of block b of a panel held row-major in P (stride S), by one warp
// (lane c = column 32 b + c): left-looking against the factored columns
// before the block (Lc: the factor, row-major stride S), then the block
// solve with the block inverse Li.  Rows of several warps run independently.
template <class T, int S>
__device__ __forceinline__ void warp_row_block(T* P, int r, int b, int jb, const T* Lc,
                                               const T* Li) {
  const int lane = threadIdx.x & 31, c0 = 32 * b;
  T* pr = P + r * S;
  T acc = lane < jb ? pr[c0 + lane] : T(0);
  const T* lrow = Lc + (c0 + lane) * S;
  if (lane < jb)
    for (int t = 0; t < c0; t++) acc -= pr[t] * lrow[t];
  T y = T(0);
#pragma unroll
  for (int t = 0; t < 32; t++) {
    const T at = __shfl_sync(0xffffffffu, acc, t);
    if (t <= lane && t < jb) y += at * Li[lane * 33 + t];
  }
  __syncwarp();
  if (lane < jb) pr[c0 + lane] = y;
}

template <class T, int W>
__global__ void __launch_bounds__(kSubThreads) k_subpanel(const int* __restrict__ flist, int nf,
                                                          const FrontDev* __restrict__ fr,
                                                          T* __restrict__ F, int Ks,
                                                          T* __restrict__ dslot, DevError* err) {
  constexpr int S = sub_stride<W>();
  extern __shared__ __align__(16) unsigned char sub_raw[];
  T* Ds = reinterpret_cast<T*>(sub_raw);   // diagonal block -> its factor, row-major stride S
  T* Xs = Ds + W * S;                      // a 128-row block of the panel
  T* Lib = Xs + kSubRows * S;              // inverses of the 32 x 32 diagonal blocks, 32 x 33 each
  __shared__ int pre[kMaxPanelFronts + 1];
  __shared__ int badcol;
  const int tid = threadIdx.x, warp = tid >> 5, nwarp = kSubThreads / 32;
  // items per front (in parallel), then their prefix (thread 0, shared memory)
  for (int i = tid; i < nf; i += kSubThreads) {
    const FrontDev d = fr[flist[i]];
    pre[i + 1] = Ks < d.n ? 1 + (d.N - Ks - min(W, d.n - Ks) + kSubRows - 1) / kSubRows : 0;
  }
  __syncthreads();
  if (tid == 0) {
    pre[0] = 0;
    for (int i = 0; i < nf; i++) pre[i + 1] += pre[i];
  }
  __syncthreads();
  const int total = pre[nf];
  int cur = -1;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    int lo = 0, hi = nf - 1;   // largest i with pre[i] <= item
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    const int i = lo, f = flist[i];
    const FrontDev d = fr[f];
    T* A = F + d.off;
    const int64_t ld = d.ld;
    const int kb = min(W, d.n - Ks), nb = (kb + 31) / 32;
    if (i != cur) {
      // load the diagonal block and factor it, 32 columns at a time, left-looking
      cur = i;
      __syncthreads();
      for (int idx = tid; idx < kb * kb; idx += kSubThreads) {
        const int r = idx % kb, c = idx / kb;
        Ds[r * S + c] = r >= c ? A[(Ks + r) + (int64_t)(Ks + c) * ld] : T(0);
      }
      if (tid == 0) badcol = -1;
      __syncthreads();
      for (int b = 0; b < nb; b++) {
        const int c0 = 32 * b, jb = min(32, kb - c0);
        // block b's diagonal block less the earlier columns' contributions
        if (b > 0)
          for (int r = c0 + warp; r < c0 + jb; r += nwarp) {
            const int lane = tid & 31;
            if (lane < jb && lane <= r - c0) {
              T acc = Ds[r * S + c0 + lane];
              const T* lr = Ds + r * S;
              const T* lc = Ds + (c0 + lane) * S;
              for (int t = 0; t < c0; t++) acc -= lr[t] * lc[t];
              Ds[r * S + c0 + lane] = acc;
            }
          }
        __syncthreads();
        if (warp == 0) {
          const int bad = warp_chol_inv<T, S>(Ds, c0, jb, Lib + b * 32 * 33);
          if ((tid & 31) == 0 && bad >= 0 && badcol < 0) badcol = Ks + c0 + bad;
        }
        __syncthreads();
        // the rows of the diagonal block below block b
        for (int r = c0 + jb + warp; r < kb; r += nwarp)
          warp_row_block<T, S>(Ds, r, b, jb, Ds, Lib + b * 32 * 33);
        __syncthreads();
      }
      if (tid == 0 && badcol >= 0 && atomicCAS(&err->code, 0, 1) == 0) {
        err->front = f;
        err->col = badcol;
      }
    }
    const int local = item - pre[i];
    if (local == 0) {   // the factored diagonal block to the front's slot
      T* slot = dslot + (int64_t)i * W * W;
      for (int idx = tid; idx < kb * kb; idx += kSubThreads) {
        const int r = idx % kb, c = idx / kb;
        if (r >= c) slot[r + c * W] = Ds[r * S + c];
      }
      continue;
    }
    const int r0 = Ks + kb + (local - 1) * kSubRows, rows = min(kSubRows, d.N - r0);
    __syncthreads();
    for (int idx = tid; idx < kSubRows * kb; idx += kSubThreads) {
      const int r = idx % kSubRows, c = idx / kSubRows;
      Xs[r * S + c] = r < rows ? A[(r0 + r) + (int64_t)(Ks + c) * ld] : T(0);
    }
    __syncthreads();
    // X <- X L^{-T}: each row by one warp, block by block, no block barrier
    for (int r = warp; r < rows; r += nwarp)
      for (int b = 0; b < nb; b++)
        warp_row_block<T, S>(Xs, r, b, min(32, kb - 32 * b), Ds, Lib + b * 32 * 33);
    __syncthreads();
    for (int idx = tid; idx < kSubRows * kb; idx += kSubThreads) {
      const int r = idx % kSubRows, c = idx / kSubRows;
      if (r < rows) A[(r0 + r) + (int64_t)(Ks + c) * ld] = Xs[r * S + c];
    }
  }
}

// The factored diagonal blocks from their slots into the fronts, a CTA per front.
template <class T, int W>
__global__ void __launch_bounds__(kSubThreads) k_panel_diag(const int* __restrict__ flist,
                                                            const FrontDev* __restrict__ fr,
                                                            T* __restrict__ F, int Ks,
                                                            const T* __restrict__ dslot) {
  const FrontDev d = fr[flist[blockIdx.x]];
  if (Ks >= d.n) return;
  const int kb = min(W, d.n - Ks);
  const T* slot = dslot + (int64_t)blockIdx.x * W * W;
  T* A = F + d.off;
  for (int idx = threadIdx.x; idx < kb * kb; idx += kSubThreads) {
    const int r = idx % kb, c = idx / kb;
    if (r >= c) A[(Ks + r) + (int64_t)(Ks + c) * d.ld] = slot[r + c * W];
  }
}

template <class T, int W>
cudaError_t launchSub(const int* flist, int nf, const FrontDev* fr, T* F, int Ks, T* dslot,
                      DevError* err, cudaStream_t st) {
  static const int grid = []() {   // thread-safe one-time set-up: every resident CTA
    int dev = 0, n = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_subpanel<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sub_smem<T, W>());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_subpanel<T, W>, kSubThreads,
                                                  sub_smem<T, W>());
    return n * std::max(1, per);
  }();
  k_subpanel<T, W><<<grid, kSubThreads, sub_smem<T, W>(), st>>>(flist, nf, fr, F, Ks, dslot, err);
  k_panel_diag<T, W><<<nf, kSubThreads, 0, st>>>(flist, fr, F, Ks, dslot);
  g_launches += 2;
  return cudaGetLastError();
}

}  // namespace

int panel_width(int elem_bytes) { return elem_bytes == 8 ? kPanelW64 : kPanelW32; }

size_t panel_slot_bytes(int nf, int elem_bytes) {
  const size_t w = (size_t)panel_width(elem_bytes);
  return (size_t)std::min(nf, kMaxPanelFronts) * w * w * (size_t)elem_bytes;
}

template <>
cudaError_t launch_subpanel<float>(const int* flist, int nf, const FrontDev* fr, float* F, int Ks,
                                   int w, float* dslot, DevError* err, cudaStream_t st) {
  if (nf <= 0) return cudaSuccess;
  if (nf > kMaxPanelFronts || w != kPanelW32 || !dslot) return cudaErrorInvalidValue;
  return launchSub<float, kPanelW32>(flist, nf, fr, F, Ks, dslot, err, st);
}
template <>
cudaError_t launch_subpanel<double>(const int* flist, int nf, const FrontDev* fr, double* F, int Ks,
                                    int w, double* dslot, DevError* err, cudaStream_t st) {
  if (nf <= 0) return cudaSuccess;
  if (nf > kMaxPanelFronts || w != kPanelW64 || !dslot) return cudaErrorInvalidValue;
  return launchSub<double, kPanelW64>(flist, nf, fr, F, Ks, dslot, err, st);
}

}  // namespace mfgpu
