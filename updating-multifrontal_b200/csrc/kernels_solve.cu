// Cooperative forward / backward sweeps for the levels of large fronts.
//
// The one-CTA-per-front sweeps (kernels_front.cu) serialise a front's whole
// triangular solve on one SM, which leaves a level of a few large fronts (the
// top of a 3D tree, the root of every problem) far below HBM bandwidth.  These
// kernels spread every front of a level over all SMs with one cooperative
// launch and a blocked, right-looking substitution over 64-column blocks:
//
//   forward  (src/DE/mf2d.cpp:976-1014, the per-box L11 solve and the
//   boundary update b_bd -= L21 y):
//     step j: every CTA with work forms y_j = L_jj^{-1} w_j from the block's
//             explicit inverse, takes 256 rows below block j and applies
//             W(rows) -= L(rows, block j) y_j; grid barrier.
//   backward (src/DE/mf2d.cpp:1016-1054, x_piv = L11^{-T}(y - L21^T x_bd)):
//     first r = y - L21^T x_bd by column blocks; then for j = last .. 0 every
//     CTA with work forms x_j = L_jj^{-T} r_j, takes one column block c < j and
//     applies r_c -= L(block j, block c)^T x_j; grid barrier.
// The inverses (k_diag_inv, after each factorization of the level) take the
// sequential substitution out of every step: a step costs one block product,
// one pass over a panel and one grid barrier.
//
// Each front's L is read once per sweep.  W is the front's right-hand-side
// block (N x nrhs, ld N) in the same workspace the per-front kernels use, so
// the separator gathers between levels are unchanged; the solved pivot blocks
// go to the second half of that workspace (another N x nrhs), so no step reads
// what another CTA of the same step writes.
#include <cooperative_groups.h>

#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace cg = cooperative_groups;

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int SB = 64;          // diagonal block of the substitution
constexpr int SCT = 256;        // threads per CTA
constexpr int kMaxSolveCoopFronts = SCT;

__host__ __device__ __forceinline__ int cdiv(int a, int b) { return (a + b - 1) / b; }

// pre[0..nf] = exclusive prefix of the per-front counts (thread t holds front
// t's count); every thread must call.
__device__ void scan_counts(int v, int nf, int* pre, int* wt) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();   // pre / wt may still be read by the previous step
  if (lane == 31) wt[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = lane < SCT / 32 ? wt[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < SCT / 32) wt[lane] = t;
  }
  __syncthreads();
  if (tid < nf) pre[tid + 1] = (w > 0 ? wt[w - 1] : 0) + x;
  if (tid == 0) pre[0] = 0;
  __syncthreads();
}

__device__ __forceinline__ int find_front(const int* pre, int nf, int item) {
  int lo = 0, hi = nf - 1;   // largest i with pre[i] <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Diagonal-block inverses of the cooperative levels' pivot blocks: block b of
// front f (rows and columns [64 b, 64 b + kb)) gets Dinv = L_bb^{-1} (lower,
// column-major 64 x 64, zero outside kb x kb) at Dv + dinv_off[f] + b * 8192
// and its transpose right after it.  Column t of the inverse is computed by
// thread t with forward substitution on the block staged in shared memory.
template <class T>
__global__ void __launch_bounds__(SB) k_diag_inv(const int* __restrict__ flist,
                                                 const FrontDev* __restrict__ fr,
                                                 const T* __restrict__ F, T* __restrict__ Dv,
                                                 const int64_t* __restrict__ dinv_off) {
  extern __shared__ __align__(16) unsigned char dsm[];   // Ls and Iv, 2 x 64 x 65
  T(*Ls)[SB + 1] = reinterpret_cast<T(*)[SB + 1]>(dsm);
  T(*Iv)[SB + 1] = Ls + SB;
  const int f = flist[blockIdx.y];
  const FrontDev d = fr[f];
  const int b = blockIdx.x, k = b * SB;
  if (k >= d.n || dinv_off[f] < 0) return;
  const int kb = min(SB, d.n - k), t = threadIdx.x;
  const T* A = F + d.off;
  for (int c = 0; c < kb; c++)
    if (t < kb) Ls[t][c] = t >= c ? A[(k + t) + (int64_t)(k + c) * d.ld] : T(0);
  __syncthreads();
  if (t < kb) {
    for (int i = 0; i < t; i++) Iv[i][t] = T(0);
    for (int i = t; i < kb; i++) {
      T acc = i == t ? T(1) : T(0);
      for (int q = t; q < i; q++) acc = fma(-Ls[i][q], Iv[q][t], acc);
      Iv[i][t] = acc / Ls[i][i];
    }
  }
  __syncthreads();
  T* D = Dv + dinv_off[f] + (int64_t)b * 2 * SB * SB;
  for (int c = 0; c < SB; c++) {
    const int r = t;
    D[r + c * SB] = (r < kb && c < kb) ? Iv[r][c] : T(0);                 // Dinv
    D[SB * SB + r + c * SB] = (r < kb && c < kb) ? Iv[c][r] : T(0);       // Dinv^T
  }
}

template <class T, int NR>
__global__ void __launch_bounds__(SCT) k_solve_coop_fwd(const int* __restrict__ flist, int nf,
                                                        const FrontDev* __restrict__ fr,
                                                        const T* __restrict__ F,
                                                        const int* __restrict__ dofs, T* X,
                                                        int64_t ldx, int nrhs, T* Wb,
                                                        const int64_t* __restrict__ woff,
                                                        int maxnb, const T* __restrict__ Dv,
                                                        const int64_t* __restrict__ dinv_off,
                                                        unsigned* gbar, DevError* err) {
  unsigned gtarget = 0;
  __shared__ int pre[kMaxSolveCoopFronts + 1];
  __shared__ int wt[SCT / 32];
  __shared__ T ws[SB][NR + 1];
  __shared__ T ys[SB][NR + 1];
  extern __shared__ __align__(16) unsigned char dsm[];
  T* Ds = reinterpret_cast<T*>(dsm);   // the step's block inverse, SB x SB
  const int tid = threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * SCT;
  // gather: pivot rows from X, boundary rows zero
  for (int i = 0; i < nf; i++) {
    const int f = flist[i];
    const FrontDev d = fr[f];
    T* W = Wb + woff[f] * nrhs;
    const int* dl = dofs + d.dof_off;
    for (int64_t idx = (int64_t)blockIdx.x * SCT + tid; idx < (int64_t)d.N * nrhs; idx += gstride) {
      const int r = (int)(idx % d.N), c = (int)(idx / d.N);
      W[idx] = r < d.n ? X[dl[r] + (int64_t)c * ldx] : T(0);
    }
  }
  grid_barrier(gbar, gtarget, err);
  for (int j = 0; j < maxnb; j++) {
    int cnt = 0;
    if (tid < nf) {
      const FrontDev d = fr[flist[tid]];
      const int k = j * SB;
      if (k < d.n) cnt = max(1, cdiv(d.N - k - min(SB, d.n - k), SCT));
    }
    scan_counts(cnt, nf, pre, wt);
    for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
      const int i = find_front(pre, nf, item);
      const int f = flist[i];
      const FrontDev d = fr[f];
      const T* A = F + d.off;
      T* W = Wb + woff[f] * nrhs;          // right-hand sides being reduced
      T* Y = W + (int64_t)d.N * nrhs;      // solved pivot blocks
      const int k = j * SB, kb = min(SB, d.n - k);
      const int local = item - pre[i];
      const int r0 = k + kb + local * SCT;
      // y_j = Dinv_j w_j (w_j is final: every block above it was applied)
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int t = idx % SB, c = idx / SB;
        ws[t][c] = t < kb ? W[k + t + (int64_t)c * d.N] : T(0);
      }
      __syncthreads();
      const T* Dj = Dv + dinv_off[f] + (int64_t)j * 2 * SB * SB;
      for (int idx = tid; idx < SB * SB; idx += SCT) Ds[idx] = Dj[idx];   // one coalesced pass
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int t = idx % SB, c = idx / SB;
        T acc = T(0);
        for (int q = 0; q <= t && q < kb; q++) acc = fma(Ds[t + q * SB], ws[q][c], acc);
        ys[t][c] = t < kb ? acc : T(0);
      }
      __syncthreads();
      if (local == 0)
        for (int idx = tid; idx < kb * nrhs; idx += SCT) {
          const int t = idx % kb, c = idx / kb;
          Y[k + t + (int64_t)c * d.N] = ys[t][c];
        }
      // rows below block j: W(r) -= L(r, block j) y_j
      const int r = r0 + tid;
      if (r < d.N) {
        T acc[NR];
#pragma unroll
        for (int c = 0; c < NR; c++) acc[c] = T(0);
        const T* Lr = A + r + (int64_t)k * d.ld;
        if (kb == SB) {
#pragma unroll
          for (int t0 = 0; t0 < SB; t0 += 16) {
            T l[16];
#pragma unroll
            for (int t = 0; t < 16; t++) l[t] = Lr[(int64_t)(t0 + t) * d.ld];
#pragma unroll
            for (int t = 0; t < 16; t++)
#pragma unroll
              for (int c = 0; c < NR; c++) acc[c] = fma(l[t], ys[t0 + t][c], acc[c]);
          }
        } else {
          for (int t = 0; t < kb; t++) {
            const T l = Lr[(int64_t)t * d.ld];
#pragma unroll
            for (int c = 0; c < NR; c++) acc[c] = fma(l, ys[t][c], acc[c]);
          }
        }
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) W[r + (int64_t)c * d.N] -= acc[c];
      }
    }
    grid_barrier(gbar, gtarget, err);
  }
  // pivots back to X; the boundary part stays in W for the separator gather
  for (int i = 0; i < nf; i++) {
    const int f = flist[i];
    const FrontDev d = fr[f];
    const T* Y = Wb + woff[f] * nrhs + (int64_t)d.N * nrhs;
    const int* dl = dofs + d.dof_off;
    for (int64_t idx = (int64_t)blockIdx.x * SCT + tid; idx < (int64_t)d.n * nrhs; idx += gstride) {
      const int r = (int)(idx % d.n), c = (int)(idx / d.n);
      X[dl[r] + (int64_t)c * ldx] = Y[r + (int64_t)c * d.N];
    }
  }
}

template <class T, int NR>
__global__ void __launch_bounds__(SCT) k_solve_coop_bwd(const int* __restrict__ flist, int nf,
                                                        const FrontDev* __restrict__ fr,
                                                        const T* __restrict__ F,
                                                        const int* __restrict__ dofs, T* X,
                                                        int64_t ldx, int nrhs, T* Wb,
                                                        const int64_t* __restrict__ woff,
                                                        int maxnb, const T* __restrict__ Dv,
                                                        const int64_t* __restrict__ dinv_off,
                                                        unsigned* gbar, DevError* err) {
  unsigned gtarget = 0;
  __shared__ int pre[kMaxSolveCoopFronts + 1];
  __shared__ int wt[SCT / 32];
  __shared__ T ws[SB][NR + 1];
  __shared__ T xj[SB][NR + 1];
  extern __shared__ __align__(16) unsigned char dsm[];
  T* Ds = reinterpret_cast<T*>(dsm);   // the step's block inverse (transposed), SB x SB
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t gstride = (int64_t)gridDim.x * SCT;
  for (int i = 0; i < nf; i++) {
    const int f = flist[i];
    const FrontDev d = fr[f];
    T* W = Wb + woff[f] * nrhs;
    const int* dl = dofs + d.dof_off;
    for (int64_t idx = (int64_t)blockIdx.x * SCT + tid; idx < (int64_t)d.N * nrhs; idx += gstride) {
      const int r = (int)(idx % d.N), c = (int)(idx / d.N);
      W[idx] = X[dl[r] + (int64_t)c * ldx];
    }
  }
  grid_barrier(gbar, gtarget, err);
  // r = y - L21^T x_bd, one column block per item
  {
    int cnt = 0;
    if (tid < nf) {
      const FrontDev d = fr[flist[tid]];
      cnt = d.m > 0 ? cdiv(d.n, SB) : 0;
    }
    scan_counts(cnt, nf, pre, wt);
    for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
      const int i = find_front(pre, nf, item);
      const int f = flist[i];
      const FrontDev d = fr[f];
      const T* A = F + d.off;
      T* W = Wb + woff[f] * nrhs;
      const int cb = item - pre[i], k = cb * SB, kb = min(SB, d.n - k);
      for (int jj = warp; jj < kb; jj += SCT / 32) {
        const T* Lc = A + (int64_t)(k + jj) * d.ld;
        T acc[NR];
#pragma unroll
        for (int c = 0; c < NR; c++) acc[c] = T(0);
        int r = d.n + lane;
        for (; r + 96 < d.N; r += 128) {
          const T l0 = Lc[r], l1 = Lc[r + 32], l2 = Lc[r + 64], l3 = Lc[r + 96];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) {
              const T* w = W + (int64_t)c * d.N + r;
              acc[c] = fma(l0, w[0], acc[c]);
              acc[c] = fma(l1, w[32], acc[c]);
              acc[c] = fma(l2, w[64], acc[c]);
              acc[c] = fma(l3, w[96], acc[c]);
            }
        }
        for (; r < d.N; r += 32) {
          const T l = Lc[r];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) acc[c] = fma(l, W[r + (int64_t)c * d.N], acc[c]);
        }
#pragma unroll
        for (int c = 0; c < NR; c++) {
          T v = acc[c];
          for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
          if (lane == 0 && c < nrhs) W[k + jj + (int64_t)c * d.N] -= v;
        }
      }
    }
    grid_barrier(gbar, gtarget, err);
  }
  // step t: front i finishes its block j = nb_i - 1 - t: x_j = Dinv_j^T r_j
  // (r_j is final), written once, and applied to every earlier column block
  for (int t = 0; t < maxnb; t++) {
    int cnt = 0;
    if (tid < nf) {
      const int j = cdiv(fr[flist[tid]].n, SB) - 1 - t;
      cnt = j >= 1 ? j : (j == 0 ? 1 : 0);
    }
    scan_counts(cnt, nf, pre, wt);
    for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
      const int i = find_front(pre, nf, item);
      const int f = flist[i];
      const FrontDev d = fr[f];
      const T* A = F + d.off;
      T* W = Wb + woff[f] * nrhs;
      T* Y = W + (int64_t)d.N * nrhs;
      const int j = cdiv(d.n, SB) - 1 - t;
      const int kj = j * SB, kbj = min(SB, d.n - kj);
      const int cb = item - pre[i], k = cb * SB;
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int r = idx % SB, c = idx / SB;
        ws[r][c] = r < kbj ? W[kj + r + (int64_t)c * d.N] : T(0);
      }
      __syncthreads();
      const T* DjT = Dv + dinv_off[f] + (int64_t)j * 2 * SB * SB + SB * SB;
      for (int idx = tid; idx < SB * SB; idx += SCT) Ds[idx] = DjT[idx];  // one coalesced pass
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int r = idx % SB, c = idx / SB;
        T acc = T(0);
        for (int q = r; q < kbj; q++) acc = fma(Ds[r + q * SB], ws[q][c], acc);
        xj[r][c] = r < kbj ? acc : T(0);
      }
      __syncthreads();
      if (cb == 0)
        for (int idx = tid; idx < kbj * nrhs; idx += SCT) {
          const int r = idx % kbj, c = idx / kbj;
          Y[kj + r + (int64_t)c * d.N] = xj[r][c];
        }
      if (j == 0) continue;
      // thread (cl, q): column k + cl of block cb, rows kj + 16 q .. +16; the
      // four row quarters of a column sit in adjacent lanes
      const int cl = tid >> 2, q = tid & 3, col = k + cl;
      T acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = T(0);
      const T* Lc = A + (int64_t)col * d.ld + kj + q * 16;
#pragma unroll
      for (int rr = 0; rr < 16; rr++) {
        const int r = q * 16 + rr;
        if (r < kbj) {
          const T l = Lc[rr];
#pragma unroll
          for (int c = 0; c < NR; c++) acc[c] = fma(l, xj[r][c], acc[c]);
        }
      }
#pragma unroll
      for (int c = 0; c < NR; c++) {
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
      }
      if (q == 0)
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) W[col + (int64_t)c * d.N] -= acc[c];
    }
    grid_barrier(gbar, gtarget, err);
  }
  for (int i = 0; i < nf; i++) {
    const int f = flist[i];
    const FrontDev d = fr[f];
    const T* Y = Wb + woff[f] * nrhs + (int64_t)d.N * nrhs;
    const int* dl = dofs + d.dof_off;
    for (int64_t idx = (int64_t)blockIdx.x * SCT + tid; idx < (int64_t)d.n * nrhs; idx += gstride) {
      const int r = (int)(idx % d.n), c = (int)(idx / d.n);
      X[dl[r] + (int64_t)c * ldx] = Y[r + (int64_t)c * d.N];
    }
  }
}

// One CTA per SM: a step's work (at most a few hundred row or column blocks)
// needs no more, and a smaller grid makes each grid barrier cheaper.
template <class K>
int coopGrid(K kern, int dyn) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, SCT, dyn);
  return per > 0 ? sms : 1;
}

template <class T, int NR>
cudaError_t launchCoopSolve(bool fwd, const int* flist, int nf, int maxn, const FrontDev* fr,
                            const T* F, const int* dofs, T* X, int64_t ldx, int nrhs, T* W,
                            const int64_t* woff, const T* Dv, const int64_t* dinv_off,
                            unsigned* gbar, DevError* err, cudaStream_t st) {
  cudaError_t me = cudaMemsetAsync(gbar, 0, sizeof(unsigned), st);
  if (me != cudaSuccess) return me;
  const int dyn = SB * SB * (int)sizeof(T);
  static const int gf = coopGrid(k_solve_coop_fwd<T, NR>, dyn);   // thread-safe one-time set-up
  static const int gb = coopGrid(k_solve_coop_bwd<T, NR>, dyn);
  int maxnb = cdiv(maxn, SB);
  void* args[] = {(void*)&flist, (void*)&nf,   (void*)&fr,   (void*)&F,
                  (void*)&dofs,  (void*)&X,    (void*)&ldx,  (void*)&nrhs,
                  (void*)&W,     (void*)&woff, (void*)&maxnb, (void*)&Dv,
                  (void*)&dinv_off, (void*)&gbar, (void*)&err};
  g_launches++;
  if (fwd)
    return cudaLaunchCooperativeKernel((const void*)k_solve_coop_fwd<T, NR>, dim3(gf), dim3(SCT),
                                       args, dyn, st);
  return cudaLaunchCooperativeKernel((const void*)k_solve_coop_bwd<T, NR>, dim3(gb), dim3(SCT), args,
                                     dyn, st);
}

}  // namespace

int solve_coop_max_fronts() { return kMaxSolveCoopFronts; }

template <class T>
cudaError_t launch_solve_coop(bool forward, const int* flist, int nf, int maxn, const FrontDev* fr,
                              const T* F, const int* dofs, T* X, int64_t ldx, int nrhs, T* W,
                              const int64_t* woff, const T* Dv, const int64_t* dinv_off,
                              unsigned* gbar, DevError* err, cudaStream_t st) {
  if (nf <= 0) return cudaSuccess;
  if (nf > kMaxSolveCoopFronts || nrhs > 16) return cudaErrorInvalidValue;
  if (nrhs == 1)
    return launchCoopSolve<T, 1>(forward, flist, nf, maxn, fr, F, dofs, X, ldx, nrhs, W, woff, Dv, dinv_off, gbar, err, st);
  if (nrhs <= 4)
    return launchCoopSolve<T, 4>(forward, flist, nf, maxn, fr, F, dofs, X, ldx, nrhs, W, woff, Dv, dinv_off, gbar, err, st);
  if (nrhs <= 8)
    return launchCoopSolve<T, 8>(forward, flist, nf, maxn, fr, F, dofs, X, ldx, nrhs, W, woff, Dv, dinv_off, gbar, err, st);
  return launchCoopSolve<T, 16>(forward, flist, nf, maxn, fr, F, dofs, X, ldx, nrhs, W, woff, Dv, dinv_off, gbar, err, st);
}

template <class T>
void launch_diag_inv(const int* flist, int nf, int maxn, const FrontDev* fr, const T* F, T* Dv,
                     const int64_t* dinv_off, cudaStream_t st) {
  if (nf <= 0 || maxn <= 0) return;
  const int sm = 2 * SB * (SB + 1) * (int)sizeof(T);
  static const bool attr = (cudaFuncSetAttribute(k_diag_inv<T>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm),
                            true);
  (void)attr;
  k_diag_inv<T><<<dim3(cdiv(maxn, SB), nf), SB, sm, st>>>(flist, fr, F, Dv, dinv_off);
  g_launches++;
}

template cudaError_t launch_solve_coop<double>(bool, const int*, int, int, const FrontDev*,
                                               const double*, const int*, double*, int64_t, int,
                                               double*, const int64_t*, const double*,
                                               const int64_t*, unsigned*, DevError*, cudaStream_t);
template cudaError_t launch_solve_coop<float>(bool, const int*, int, int, const FrontDev*,
                                              const float*, const int*, float*, int64_t, int, float*,
                                              const int64_t*, const float*, const int64_t*,
                                              unsigned*, DevError*, cudaStream_t);
template void launch_diag_inv<double>(const int*, int, int, const FrontDev*, const double*, double*,
                                      const int64_t*, cudaStream_t);
template void launch_diag_inv<float>(const int*, int, int, const FrontDev*, const float*, float*,
                                     const int64_t*, cudaStream_t);

}  // namespace mfgpu
