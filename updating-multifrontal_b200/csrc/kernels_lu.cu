// Pivoted LU of the fronts of nonsymmetric problems (separator width 2-3), FP64.
//
// The reference factors every front's pivot block with LAPACK's partial-
// pivoting LU (dgetrf on A22, include/LinAlg/dense.hpp:180-188) and forms
//     XL = A12 A22^{-1},  XR = A22^{-1} A21,  S = -A12 XR
// (src/DE/mf2d.cpp:558-567).  Here each front is stored whole (column-major,
// pivots first: [A22 A21; A12 A11]) and factored in place, right-looking, in
// 32-column steps k:
//   k_lu_panel       one CTA per front: columns [k, k + kb) over rows [k, N),
//                    pivots chosen among the pivot rows [j, n) only (the
//                    boundary rows are eliminated, never swapped, as in the
//                    reference where A12 is outside dgetrf's matrix), row
//                    swaps inside the panel, multipliers, in-panel update;
//   k_lu_swap_trsm   the panel's row swaps applied to every other column (the
//                    L columns on the left too, LAPACK's convention, so that a
//                    solve applies all swaps first), then U(k block, right) =
//                    L_kk^{-1} (...) for the columns right of the panel;
//   k_lu_gemm        A(k1:N, k1:N) -= L(k1:N, k:k1) U(k:k1, k1:N) in 64 x 64
//                    tiles on the FP64 tensor cores (mma.sync m8n8k4).
// On exit rows/cols [0,n) hold L11 (unit lower) and U11 with P A22 = L11 U11,
// rows [n,N) x cols [0,n) hold L21 = A12 U11^{-1}, rows [0,n) x cols [n,N)
// hold U12 = L11^{-1} P A21 and the trailing block S + A11.  So XL = L21
// L11^{-1} P and XR = U11^{-1} U12, and the solve / apply sweeps
// (kernels_front.cu) use the factors directly.  ipiv[j] (front-relative row)
// is stored beside the front's pivot DOFs.  A zero pivot column (the pivot
// block is singular) records error code 4.
#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int kLuPanelThreads = 256;
constexpr int kLuSwapThreads = 128;
constexpr int kLuTile = 64;
constexpr int kLuS = 36;   // shared-memory row stride (doubles) of a staged tile operand

__device__ __forceinline__ void lu_report(DevError* err, int code, int front, int col) {
  if (atomicCAS(&err->code, 0, code) == 0) {
    err->front = front;
    err->col = col;
  }
}

// Panel factorization with partial pivoting restricted to the pivot rows.
__global__ void __launch_bounds__(kLuPanelThreads) k_lu_panel(const int* __restrict__ flist,
                                                              const FrontDev* __restrict__ fr,
                                                              double* __restrict__ F,
                                                              int* __restrict__ ipiv, int k,
                                                              DevError* err) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  if (k >= d.n) return;
  const int kb = min(kPanel, d.n - k), tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* A = F + d.off;
  const int64_t ld = d.ld;
  __shared__ double rowj[kPanel];
  __shared__ double wbest[kLuPanelThreads / 32];
  __shared__ int widx[kLuPanelThreads / 32];
  __shared__ int piv;
  for (int jj = 0; jj < kb; jj++) {
    const int j = k + jj;
    // pivot: the first row of largest magnitude in column j among rows [j, n)
    double best = -1.0;
    int bi = d.n;
    for (int i = j + tid; i < d.n; i += kLuPanelThreads) {
      const double v = fabs(A[i + (int64_t)j * ld]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      wbest[warp] = best;
      widx[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double b = wbest[0];
      int p = widx[0];
      for (int w = 1; w < kLuPanelThreads / 32; w++)
        if (wbest[w] > b || (wbest[w] == b && widx[w] < p)) {
          b = wbest[w];
          p = widx[w];
        }
      if (!(b > 0.0) || p >= d.n) {   // zero (or NaN) column: the pivot block is singular
        lu_report(err, 4, f, j);
        p = j;
      }
      piv = p;
      ipiv[d.dof_off + j] = p;
    }
    __syncthreads();
    const int p = piv;
    if (p != j && tid < kb) {
      double* a = A + (int64_t)(k + tid) * ld;
      const double t = a[j];
      a[j] = a[p];
      a[p] = t;
    }
    __syncthreads();
    if (tid < kb) rowj[tid] = A[j + (int64_t)(k + tid) * ld];
    __syncthreads();
    const double djj = rowj[jj];
    const double r = djj != 0.0 ? 1.0 / djj : 0.0;
    for (int i = j + 1 + tid; i < d.N; i += kLuPanelThreads) {
      const double l = A[i + (int64_t)j * ld] * r;
      A[i + (int64_t)j * ld] = l;
      for (int t = jj + 1; t < kb; t++) A[i + (int64_t)(k + t) * ld] -= l * rowj[t];
    }
    __syncthreads();
  }
}

// Row swaps of panel k on every column outside the panel, then the unit-lower
// triangular solve of the block row for the columns right of it.
__global__ void __launch_bounds__(kLuSwapThreads) k_lu_swap_trsm(const int* __restrict__ flist,
                                                                 const FrontDev* __restrict__ fr,
                                                                 double* __restrict__ F,
                                                                 const int* __restrict__ ipiv,
                                                                 int k) {
  const FrontDev d = fr[flist[blockIdx.y]];
  if (k >= d.n) return;
  const int kb = min(kPanel, d.n - k), k1 = k + kb;
  double* A = F + d.off;
  const int64_t ld = d.ld;
  __shared__ double L[kPanel][kPanel + 1];
  __shared__ int pv[kPanel];
  for (int idx = threadIdx.x; idx < kb * kb; idx += kLuSwapThreads) {
    const int i = idx % kb, j = idx / kb;
    L[i][j] = A[(k + i) + (int64_t)(k + j) * ld];
  }
  if (threadIdx.x < kb) pv[threadIdx.x] = ipiv[d.dof_off + k + threadIdx.x] - k;
  __syncthreads();
  const int c = blockIdx.x * kLuSwapThreads + threadIdx.x;
  if (c >= d.N || (c >= k && c < k1)) return;
  double* col = A + (int64_t)c * ld;
  double x[kPanel];
#pragma unroll
  for (int t = 0; t < kPanel; t++) x[t] = t < kb ? col[k + t] : 0.0;
  for (int j = 0; j < kb; j++) {
    const int p = pv[j];
    if (p == j) continue;
    if (p < kb) {
      const double t = x[j];
      x[j] = x[p];
      x[p] = t;
    } else {
      const double t = col[k + p];
      col[k + p] = x[j];
      x[j] = t;
    }
  }
  if (c >= k1) {
#pragma unroll
    for (int i = 1; i < kPanel; i++) {
      if (i < kb) {
        double s = x[i];
#pragma unroll
        for (int j = 0; j < i; j++) s -= L[i][j] * x[j];
        x[i] = s;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    if (t < kb) col[k + t] = x[t];
}

__device__ __forceinline__ void lu_dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Trailing update of step k, one 64 x 64 tile per CTA: blockIdx.x = tile of
// the front's (N - k1)^2 block (row-block fastest), blockIdx.y = front slot.
// Four warps each own a 32 x 32 quarter in the m8n8k4 accumulator layout.
__global__ void __launch_bounds__(128) k_lu_gemm(const int* __restrict__ flist,
                                                 const FrontDev* __restrict__ fr,
                                                 double* __restrict__ F, int k) {
  const FrontDev d = fr[flist[blockIdx.y]];
  if (k >= d.n) return;
  const int kb = min(kPanel, d.n - k), k1 = k + kb, R = d.N - k1;
  const int nt = (R + kLuTile - 1) / kLuTile;
  if ((int)blockIdx.x >= nt * nt) return;
  const int r0 = k1 + (blockIdx.x % nt) * kLuTile, c0 = k1 + (blockIdx.x / nt) * kLuTile;
  double* A = F + d.off;
  const int64_t ld = d.ld;
  __shared__ double Xa[kLuTile * kLuS];   // Xa[i][t] = L(r0 + i, k + t)
  __shared__ double Xb[kLuTile * kLuS];   // Xb[j][t] = U(k + t, c0 + j)
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kLuTile * kPanel; idx += 128) {
    const int i = idx % kLuTile, t = idx / kLuTile;
    Xa[i * kLuS + t] = (t < kb && r0 + i < d.N) ? A[(r0 + i) + (int64_t)(k + t) * ld] : 0.0;
  }
  for (int idx = tid; idx < kLuTile * kPanel; idx += 128) {
    const int t = idx % kPanel, j = idx / kPanel;
    Xb[j * kLuS + t] = (t < kb && c0 + j < d.N) ? A[(k + t) + (int64_t)(c0 + j) * ld] : 0.0;
  }
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5, wi = warp >> 1, wj = warp & 1;
  const int rr = lane >> 2, cc = lane & 3;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
  const int kk = (kb + 3) & ~3;
  for (int t = 0; t < kk; t += 4) {
    double fa[4], fb[4];
#pragma unroll
    for (int a = 0; a < 4; a++) fa[a] = Xa[(wi * 32 + 8 * a + rr) * kLuS + t + cc];
#pragma unroll
    for (int b = 0; b < 4; b++) fb[b] = Xb[(wj * 32 + 8 * b + rr) * kLuS + t + cc];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) lu_dmma(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
  }
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int c = c0 + wj * 32 + 8 * b + 2 * cc + q;
      if (c >= d.N) continue;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int r = r0 + wi * 32 + 8 * a + rr;
        if (r < d.N) A[r + (int64_t)c * ld] -= acc[a][b][q];
      }
    }
}

}  // namespace

void launch_lu_step(const int* flist, int nf, int maxN, const FrontDev* fr, double* F, int* ipiv,
                    int k, DevError* err, cudaStream_t st, int phase) {
  if (nf <= 0) return;
  if (phase == 0) {
    k_lu_panel<<<nf, kLuPanelThreads, 0, st>>>(flist, fr, F, ipiv, k, err);
  } else if (phase == 1) {
    const int gx = (maxN + kLuSwapThreads - 1) / kLuSwapThreads;
    k_lu_swap_trsm<<<dim3(gx, nf), kLuSwapThreads, 0, st>>>(flist, fr, F, ipiv, k);
  } else {
    const int R = maxN - k - 1;
    if (R <= 0) return;
    const int nt = (R + kLuTile - 1) / kLuTile;
    k_lu_gemm<<<dim3(nt * nt, nf), 128, 0, st>>>(flist, fr, F, k);
  }
  g_launches++;
}

}  // namespace mfgpu
