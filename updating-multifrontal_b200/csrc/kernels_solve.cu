// Cooperative forward / backward sweeps for the levels of large fronts.
//
// The one-CTA-per-front sweeps (kernels_front.cu) serialise a front's whole
// triangular solve on one SM, which leaves a level of a few large fronts (the
// top of a 3D tree, the root of every problem) far below HBM bandwidth.  These
// kernels spread every front of a level over all SMs with one persistent
// cooperative launch and a blocked substitution over 64-row blocks, ordered
// by ready flags instead of grid barriers:
//
//   forward  (src/DE/mf2d.cpp:976-1014, the per-box L11 solve and the
//   boundary update b_bd -= L21 y): a task per 64-row block of a front
//   accumulates L(block, j) y_j over the solved blocks j before it and, for a
//   pivot block, solves y = L_bb^{-1}(b - acc) with the block's explicit
//   inverse and raises the block's flag;
//   backward (src/DE/mf2d.cpp:1016-1054, x_piv = L11^{-T}(y - L21^T x_bd)): a
//   task per 64-column pivot block accumulates L(rows below, block)^T x over
//   the boundary rows and the solved blocks after it, then x = L_bb^{-T}(...)
//   and the flag.
// The inverses (k_diag_inv, after each factorization of the level) take the
// sequential substitution out of every block; the chain of dependent blocks
// costs one flag hand-off and two 64 x 64 products per block, and the rest of
// the work (every element of L read once) overlaps it.
//
// W is the front's right-hand-side block (N x nrhs, ld N) in the same
// workspace the per-front kernels use, so the separator gathers between
// levels are unchanged; the solved pivot blocks go to the second half of that
// workspace (Y, another N x nrhs), where other tasks read them.
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <vector>

#include "device.cuh"

namespace cg = cooperative_groups;

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int SB = 64;          // diagonal block of the substitution
constexpr int SCT = 256;        // threads per CTA
constexpr int kMaxSolveCoopFronts = 256;

__host__ __device__ __forceinline__ int cdiv(int a, int b) { return (a + b - 1) / b; }

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

// Ready flags of the solved pivot blocks: written once per launch (after the
// block's values are visible device-wide), read by spinning thread 0s.  A
// wait gives up after the error word's poll limit (default kFlowSpin),
// records error code 3 and lets the CTA go on, so the launch always ends.
constexpr unsigned kFlowSpin = 1u << 25;

__device__ __forceinline__ void flow_wait(const int* flag, DevError* err) {
  const volatile int* f = flag;
  volatile int* code = err ? &err->code : nullptr;
  const unsigned lim = wait_limit(err, kFlowSpin);
  unsigned it = 0;
  while (*f == 0) {
    if (++it > lim) {
      if (err) atomicCAS(&err->code, 0, 3);
      break;
    }
    if ((it & 1023u) == 0 && code && *code == 3) break;   // another CTA gave up
    __nanosleep(32);
  }
  __threadfence();
}

__device__ __forceinline__ void flow_publish(int* flag) {
  __threadfence();
  atomicExch(flag, 1);
}

template <class T>
__device__ __forceinline__ T ldcg(const T* p) {
  return __ldcg(p);
}

// Forward sweep of one level without grid barriers.  Row blocks of every
// front (pivot blocks [64 R, 64 R + 64) of [0, n), then boundary blocks of 64
// rows from n) are tasks, listed R-major across the fronts; CTAs take them
// round-robin.  Task (i, R) accumulates L(rows, block j) y_j over the pivot
// column blocks j before it as their ready flags come up, then a pivot block
// forms y_R = Dinv_R (b_R - acc), writes it to X and to the front's second
// workspace half (Y) and raises its flag; a boundary block leaves -acc in W
// for the separator gather.  Everything the last dependency does not change -
// its L block, the block's row of the inverse, the right-hand side - is in
// registers before the task waits for it, so a step of the chain of dependent
// blocks costs one small load, a product and two four-lane reductions.  The
// four lanes of a row (tid & 3) split its 64 columns; a warp's loads of one
// column offset still cover whole 32-byte sectors.  A task waits only on
// tasks listed before it, and a cooperative launch keeps every CTA resident,
// so the sweep cannot stall.
template <class T, int NR>
__global__ void __launch_bounds__(SCT) k_solve_flow_fwd(const int* __restrict__ flist,
                                                        const FrontDev* __restrict__ fr,
                                                        const T* __restrict__ F,
                                                        const int* __restrict__ dofs, T* X,
                                                        int64_t ldx, int nrhs, T* Wb,
                                                        const int64_t* __restrict__ woff,
                                                        const T* __restrict__ Dv,
                                                        const int64_t* __restrict__ dinv_off,
                                                        const int2* __restrict__ tasks, int ntasks,
                                                        const int* __restrict__ flagoff, int* flags,
                                                        DevError* err) {
  constexpr int CH = 4;                       // column blocks per shared-memory round
  __shared__ T ys[CH * SB][NR + 1];           // solved blocks
  __shared__ T ws[SB][NR + 1];                // b_R - acc of the block
  const int tid = threadIdx.x, rl = tid >> 2, g = tid & 3;   // row, column quarter
  for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
    const int2 tk = tasks[t];
    const int i = tk.x, R = tk.y, f = flist[i];
    const FrontDev d = fr[f];
    const T* A = F + d.off;
    T* W = Wb + woff[f] * nrhs;
    T* Y = W + (int64_t)d.N * nrhs;
    const int* dl = dofs + d.dof_off;
    const int* fl = flags + flagoff[i];
    const int nb = cdiv(d.n, SB);
    const bool piv = R < nb;
    const int row0 = piv ? R * SB : d.n + (R - nb) * SB;
    const int rows = min(SB, (piv ? d.n : d.N) - row0);
    const bool live = rl < rows;
    const int jmax = piv ? R : nb;
    const T* Ar = A + row0 + rl;
    T acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = T(0);
    // every block but the last, CH at a time as their flags come up.  These
    // bulk loads go by (row tid & 63, column group tid >> 6): a warp reads 32
    // consecutive rows of a column (coalesced); the sums are handed to the
    // (row, quarter) lanes once, after the loop.
    const int rl2 = tid & (SB - 1), g2 = tid >> 6;
    const T* Ar2 = A + row0 + rl2;
    T acc2[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc2[c] = T(0);
    for (int j0 = 0; j0 < jmax - 1; j0 += CH) {
      const int jc = min(CH, jmax - 1 - j0);
      __syncthreads();                        // ys of the previous round is consumed
      if (tid == 0)
        for (int jj = 0; jj < jc; jj++) flow_wait(fl + j0 + jj, err);
      __syncthreads();
      for (int idx = tid; idx < jc * SB * nrhs; idx += SCT) {
        const int r = idx % (jc * SB), c = idx / (jc * SB);
        const int col = j0 * SB + r;
        ys[r][c] = col < d.n ? ldcg(Y + col + (int64_t)c * d.N) : T(0);
      }
      __syncthreads();
      if (rl2 < rows) {
        for (int jj = 0; jj < jc; jj++) {
          const int cb = (j0 + jj) * SB + 16 * g2;
          T l[16];
#pragma unroll
          for (int q = 0; q < 16; q++) l[q] = cb + q < d.n ? Ar2[(int64_t)(cb + q) * d.ld] : T(0);
#pragma unroll
          for (int q = 0; q < 16; q++)
#pragma unroll
            for (int c = 0; c < NR; c++) acc2[c] = fma(l[q], ys[jj * SB + 16 * g2 + q][c], acc2[c]);
        }
      }
    }
    if (jmax > 1) {                           // hand the sums to the (row, quarter) lanes
      __syncthreads();
#pragma unroll
      for (int c = 0; c < NR; c++) ys[g2 * SB + rl2][c] = acc2[c];
      __syncthreads();
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = ys[g * SB + rl][c];
    }
    // before the last wait: that block's L values, this row's quarter of
    // Dinv_R (lower triangular, column-major) and the right-hand side
    T ll[16], dv[16], w[NR];
    const int cl = (jmax - 1) * SB + 16 * g;
#pragma unroll
    for (int q = 0; q < 16; q++)
      ll[q] = (jmax > 0 && live && cl + q < d.n) ? Ar[(int64_t)(cl + q) * d.ld] : T(0);
    if (piv) {
      const T* D = Dv + dinv_off[f] + (int64_t)R * 2 * SB * SB;
#pragma unroll
      for (int q = 0; q < 16; q++) dv[q] = 16 * g + q <= rl ? D[rl + (16 * g + q) * SB] : T(0);
#pragma unroll
      for (int c = 0; c < NR; c++)
        w[c] = (live && g == 0 && c < nrhs) ? X[dl[row0 + rl] + (int64_t)c * ldx] : T(0);
    }
    if (jmax > 0) {
      __syncthreads();                        // ys of the previous round is consumed
      if (tid == 0) flow_wait(fl + jmax - 1, err);
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int r = idx % SB, c = idx / SB;
        const int col = (jmax - 1) * SB + r;
        ys[r][c] = col < d.n ? ldcg(Y + col + (int64_t)c * d.N) : T(0);
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 16; q++)
#pragma unroll
        for (int c = 0; c < NR; c++) acc[c] = fma(ll[q], ys[16 * g + q][c], acc[c]);
    }
    // sum the four quarters of the row
#pragma unroll
    for (int c = 0; c < NR; c++) {
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
    }
    if (!piv) {
      if (live && g == 0)
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) W[row0 + rl + (int64_t)c * d.N] = -acc[c];
      continue;
    }
    if (g == 0)
#pragma unroll
      for (int c = 0; c < NR; c++) ws[rl][c] = live ? w[c] - acc[c] : T(0);
    __syncthreads();
    // y_R = Dinv_R w_R: each lane its quarter, then the four-lane sum
    T y[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) y[c] = T(0);
#pragma unroll
    for (int q = 0; q < 16; q++)
#pragma unroll
      for (int c = 0; c < NR; c++) y[c] = fma(dv[q], ws[16 * g + q][c], y[c]);
#pragma unroll
    for (int c = 0; c < NR; c++) {
      y[c] += __shfl_xor_sync(0xffffffffu, y[c], 1);
      y[c] += __shfl_xor_sync(0xffffffffu, y[c], 2);
    }
    if (live && g == 0)
#pragma unroll
      for (int c = 0; c < NR; c++)
        if (c < nrhs) {
          Y[row0 + rl + (int64_t)c * d.N] = y[c];
          X[dl[row0 + rl] + (int64_t)c * ldx] = y[c];
        }
    __syncthreads();
    if (tid == 0) flow_publish(flags + flagoff[i] + R);
  }
}

// Backward sweep of one level without grid barriers: x_piv = L11^{-T}
// (y - L21^T x_bd).  Task (i, j), pivot column block j of front i, listed by
// distance from the front's last block: r = sum over the rows below block j of
// L(r, block j)^T x_r, the boundary rows first (x_bd is final on entry), then
// the solved pivot blocks from the last one down as their flags come up (the
// nearest block, the last dependency, with its L values, this column's
// quarter of Dinv_j^T and y_j in registers before the wait); then
// x_j = Dinv_j^T (y_j - r) to X and Y and the flag.  The four lanes of a
// column (tid & 3) split the rows.
template <class T, int NR>
__global__ void __launch_bounds__(SCT) k_solve_flow_bwd(const int* __restrict__ flist,
                                                        const FrontDev* __restrict__ fr,
                                                        const T* __restrict__ F,
                                                        const int* __restrict__ dofs, T* X,
                                                        int64_t ldx, int nrhs, T* Wb,
                                                        const int64_t* __restrict__ woff,
                                                        const T* __restrict__ Dv,
                                                        const int64_t* __restrict__ dinv_off,
                                                        const int2* __restrict__ tasks, int ntasks,
                                                        const int* __restrict__ flagoff, int* flags,
                                                        DevError* err) {
  constexpr int BR = 4;                       // boundary row blocks per shared-memory round
  // Up to four right-hand sides the rows below go warp by column: warp wp
  // takes columns 8 wp .. 8 wp + 7 of the block, its lanes 32 consecutive rows
  // per load (coalesced), and a shuffle reduction sums the lanes at the end.
  constexpr bool CW = NR <= 4;
  __shared__ T xs[BR * SB][NR + 1];
  __shared__ T vs[SB][NR + 1];
  __shared__ T red[CW ? SB : 1][NR + 1];
  const int tid = threadIdx.x, cl = tid >> 2, q = tid & 3;   // column of the block, row quarter
  const int wl = tid & 31, wp = tid >> 5;
  for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
    const int2 tk = tasks[t];
    const int i = tk.x, j = tk.y, f = flist[i];
    const FrontDev d = fr[f];
    const T* A = F + d.off;
    T* W = Wb + woff[f] * nrhs;
    T* Y = W + (int64_t)d.N * nrhs;
    const int* dl = dofs + d.dof_off;
    const int* fl = flags + flagoff[i];
    const int nb = cdiv(d.n, SB), col0 = j * SB, kbj = min(SB, d.n - col0);
    const bool live = cl < kbj;
    const T* Lc = A + (int64_t)(col0 + cl) * d.ld;
    T acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = T(0);
    T accw[CW ? 8 : 1][NR];
#pragma unroll
    for (int k = 0; k < (CW ? 8 : 1); k++)
#pragma unroll
      for (int c = 0; c < NR; c++) accw[k][c] = T(0);
    // rows [r0, r0 + nr) (nr <= 64) against xs rows [x0, x0 + nr), every
    // load in flight before the products
    auto chunk = [&](int r0, int nr, int x0) {
      if constexpr (CW) {
        T l0[8], l1[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int c = 8 * wp + k;
          const T* Lk = A + (int64_t)(col0 + c) * d.ld + r0;
          l0[k] = (c < kbj && wl < nr) ? Lk[wl] : T(0);
          l1[k] = (c < kbj && wl + 32 < nr) ? Lk[wl + 32] : T(0);
        }
#pragma unroll
        for (int k = 0; k < 8; k++)
#pragma unroll
          for (int c = 0; c < NR; c++)
            accw[k][c] = fma(l1[k], xs[x0 + wl + 32][c], fma(l0[k], xs[x0 + wl][c], accw[k][c]));
      } else {
        // lanes (cl, q) take rows 16 q .. 16 q + 15
        if (!live) return;
        T l[16];
#pragma unroll
        for (int rr = 0; rr < 16; rr++) l[rr] = 16 * q + rr < nr ? Lc[r0 + 16 * q + rr] : T(0);
#pragma unroll
        for (int rr = 0; rr < 16; rr++)
#pragma unroll
          for (int c = 0; c < NR; c++) acc[c] = fma(l[rr], xs[x0 + 16 * q + rr][c], acc[c]);
      }
    };
    for (int r0 = d.n; r0 < d.N; r0 += BR * SB) {      // boundary rows: x_bd from X
      const int nr = min(BR * SB, d.N - r0);
      __syncthreads();
      for (int idx = tid; idx < BR * SB * nrhs; idx += SCT) {
        const int r = idx % (BR * SB), c = idx / (BR * SB);
        xs[r][c] = r < nr ? X[dl[r0 + r] + (int64_t)c * ldx] : T(0);
      }
      __syncthreads();
#pragma unroll
      for (int s = 0; s < BR; s++)
        if (s * SB < nr) chunk(r0 + s * SB, min(SB, nr - s * SB), s * SB);
    }
    for (int R = nb - 1; R > j + 1; R--) {              // solved pivot blocks below but the nearest
      const int r0 = R * SB, nr = min(SB, d.n - r0);
      __syncthreads();
      if (tid == 0) flow_wait(fl + R, err);
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int r = idx % SB, c = idx / SB;
        xs[r][c] = r < nr ? ldcg(Y + r0 + r + (int64_t)c * d.N) : T(0);
      }
      __syncthreads();
      chunk(r0, nr, 0);
    }
    if constexpr (CW) {                      // the warps' column sums to the (cl, q) lanes
#pragma unroll
      for (int k = 0; k < 8; k++)
#pragma unroll
        for (int c = 0; c < NR; c++) {
          T v = accw[k][c];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (wl == 0) red[8 * wp + k][c] = v;
        }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = (q == 0 && live) ? red[cl][c] : T(0);
    }
    // before the last wait: block j + 1's L values, this column's quarter of
    // Dinv_j^T (upper triangular, column-major) and y_j
    const int rn = (j + 1) * SB, nn = j + 1 < nb ? min(SB, d.n - rn) : 0;
    T ln[16], dt[16], v[NR];
#pragma unroll
    for (int rr = 0; rr < 16; rr++)
      ln[rr] = (live && 16 * q + rr < nn) ? Lc[rn + 16 * q + rr] : T(0);
    {
      const T* D = Dv + dinv_off[f] + (int64_t)j * 2 * SB * SB + SB * SB;
#pragma unroll
      for (int p = 0; p < 16; p++) dt[p] = 16 * q + p >= cl ? D[cl + (16 * q + p) * SB] : T(0);
#pragma unroll
      for (int c = 0; c < NR; c++)
        v[c] = (live && q == 0 && c < nrhs) ? X[dl[col0 + cl] + (int64_t)c * ldx] : T(0);
    }
    if (nn > 0) {
      __syncthreads();                        // xs of the previous round is consumed
      if (tid == 0) flow_wait(fl + j + 1, err);
      __syncthreads();
      for (int idx = tid; idx < SB * nrhs; idx += SCT) {
        const int r = idx % SB, c = idx / SB;
        xs[r][c] = r < nn ? ldcg(Y + rn + r + (int64_t)c * d.N) : T(0);
      }
      __syncthreads();
#pragma unroll
      for (int rr = 0; rr < 16; rr++)
#pragma unroll
        for (int c = 0; c < NR; c++) acc[c] = fma(ln[rr], xs[16 * q + rr][c], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < NR; c++) {
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
    }
    __syncthreads();                          // vs of the previous task is consumed
    if (q == 0)
#pragma unroll
      for (int c = 0; c < NR; c++) vs[cl][c] = live ? v[c] - acc[c] : T(0);
    __syncthreads();
    // x_j = Dinv_j^T v: each lane its quarter, then the four-lane sum
    T x[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) x[c] = T(0);
#pragma unroll
    for (int p = 0; p < 16; p++)
#pragma unroll
      for (int c = 0; c < NR; c++) x[c] = fma(dt[p], vs[16 * q + p][c], x[c]);
#pragma unroll
    for (int c = 0; c < NR; c++) {
      x[c] += __shfl_xor_sync(0xffffffffu, x[c], 1);
      x[c] += __shfl_xor_sync(0xffffffffu, x[c], 2);
    }
    if (live && q == 0)
#pragma unroll
      for (int c = 0; c < NR; c++)
        if (c < nrhs) {
          Y[col0 + cl + (int64_t)c * d.N] = x[c];
          X[dl[col0 + cl] + (int64_t)c * ldx] = x[c];
        }
    __syncthreads();
    if (tid == 0) flow_publish(flags + flagoff[i] + j);
  }
}

// Persistent grid: every CTA the SMs hold at once (a cooperative launch checks
// that they are all resident, which the flag waits rely on).  As many CTAs as
// fit, so that the row blocks of a long chain (a root front has hundreds) each
// get their own CTA from the start and accumulate the solved blocks as they
// come, instead of queueing behind other tasks of the same CTA.
template <class K>
int flowGrid(K kern) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, SCT, 0);
  return sms * std::max(1, per);
}

template <class T, int NR>
cudaError_t launchFlowSolve(bool fwd, const int* flist, const FrontDev* fr, const T* F,
                            const int* dofs, T* X, int64_t ldx, int nrhs, T* W,
                            const int64_t* woff, const T* Dv, const int64_t* dinv_off,
                            const int2* tasks, int ntasks, const int* flagoff, int* flags,
                            int nflags, DevError* err, cudaStream_t st) {
  cudaError_t me = cudaMemsetAsync(flags, 0, sizeof(int) * (size_t)std::max(1, nflags), st);
  if (me != cudaSuccess) return me;
  static const int gf = flowGrid(k_solve_flow_fwd<T, NR>);   // thread-safe one-time set-up
  static const int gb = flowGrid(k_solve_flow_bwd<T, NR>);
  const int grid = std::max(1, std::min(fwd ? gf : gb, ntasks));
  void* args[] = {(void*)&flist, (void*)&fr,    (void*)&F,      (void*)&dofs,    (void*)&X,
                  (void*)&ldx,   (void*)&nrhs,  (void*)&W,      (void*)&woff,    (void*)&Dv,
                  (void*)&dinv_off, (void*)&tasks, (void*)&ntasks, (void*)&flagoff, (void*)&flags,
                  (void*)&err};
  g_launches++;
  if (fwd)
    return cudaLaunchCooperativeKernel((const void*)k_solve_flow_fwd<T, NR>, dim3(grid), dim3(SCT),
                                       args, 0, st);
  return cudaLaunchCooperativeKernel((const void*)k_solve_flow_bwd<T, NR>, dim3(grid), dim3(SCT),
                                     args, 0, st);
}

}  // namespace

int solve_coop_max_fronts() { return kMaxSolveCoopFronts; }

void flow_tasks(const std::vector<int>& n, const std::vector<int>& N, std::vector<int>& fwd,
                std::vector<int>& bwd, std::vector<int>& flagoff) {
  const int nf = (int)n.size();
  std::vector<int> nb(nf), rb(nf);
  int maxrb = 0, maxnb = 0;
  flagoff.assign(nf + 1, 0);
  for (int i = 0; i < nf; i++) {
    nb[i] = cdiv(n[i], SB);
    rb[i] = nb[i] + cdiv(N[i] - n[i], SB);
    maxrb = std::max(maxrb, rb[i]);
    maxnb = std::max(maxnb, nb[i]);
    flagoff[i + 1] = flagoff[i] + nb[i];
  }
  fwd.clear();
  bwd.clear();
  for (int R = 0; R < maxrb; R++)
    for (int i = 0; i < nf; i++)
      if (R < rb[i]) fwd.insert(fwd.end(), {i, R});
  for (int t = 0; t < maxnb; t++)
    for (int i = 0; i < nf; i++)
      if (t < nb[i]) bwd.insert(bwd.end(), {i, nb[i] - 1 - t});
}

template <class T>
cudaError_t launch_solve_flow(bool forward, const int* flist, const FrontDev* fr, const T* F,
                              const int* dofs, T* X, int64_t ldx, int nrhs, T* W,
                              const int64_t* woff, const T* Dv, const int64_t* dinv_off,
                              const int* tasks, int ntasks, const int* flagoff, int* flags,
                              int nflags, DevError* err, cudaStream_t st) {
  if (ntasks <= 0) return cudaSuccess;
  if (nrhs > 16) return cudaErrorInvalidValue;
  const int2* tk = reinterpret_cast<const int2*>(tasks);
#define MFGPU_FLOW(NRV)                                                                           \
  return launchFlowSolve<T, NRV>(forward, flist, fr, F, dofs, X, ldx, nrhs, W, woff, Dv, dinv_off, \
                                 tk, ntasks, flagoff, flags, nflags, err, st)
  if (nrhs == 1) MFGPU_FLOW(1);
  if (nrhs <= 4) MFGPU_FLOW(4);
  if (nrhs <= 8) MFGPU_FLOW(8);
  MFGPU_FLOW(16);
#undef MFGPU_FLOW
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

template cudaError_t launch_solve_flow<double>(bool, const int*, const FrontDev*, const double*,
                                               const int*, double*, int64_t, int, double*,
                                               const int64_t*, const double*, const int64_t*,
                                               const int*, int, const int*, int*, int, DevError*,
                                               cudaStream_t);
template cudaError_t launch_solve_flow<float>(bool, const int*, const FrontDev*, const float*,
                                              const int*, float*, int64_t, int, float*,
                                              const int64_t*, const float*, const int64_t*,
                                              const int*, int, const int*, int*, int, DevError*,
                                              cudaStream_t);
template void launch_diag_inv<double>(const int*, int, int, const FrontDev*, const double*, double*,
                                      const int64_t*, cudaStream_t);
template void launch_diag_inv<float>(const int*, int, int, const FrontDev*, const float*, float*,
                                     const int64_t*, cudaStream_t);

}  // namespace mfgpu
