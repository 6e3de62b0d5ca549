// Front kernels for both precisions (T = double for the FP64 path, T = float
// for the mixed-precision factorization): front / separator assembly from
// task tables, partial Cholesky of every front of a level (fused per front, or
// one cooperative launch per level), and the solve / apply sweeps.  FP64 tiles
// use the FP64 tensor cores (mma.sync m8n8k4); FP32 tiles use CUDA-core FMAs
// with the same fragment layout.
//
// Fronts are column-major with leading dimension ld; only the lower triangle
// is read or written.  After the partial factorization of a front with n
// pivots and m boundary rows:
//   rows/cols [0,n) x [0,n)  hold L11 (A22 = L11 L11^T),
//   rows [n,N) x cols [0,n)  hold L21 (= A12 L11^{-T}),
//   rows/cols [n,N)^2        hold the update matrix: Schur complement
//                            S = -L21 L21^T on the separator diagonal blocks,
//                            A11 + S elsewhere (the reference's A11post).
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <vector>

#include "device.cuh"

namespace cg = cooperative_groups;

namespace mfgpu {

std::atomic<long long> g_launches{0};

namespace {

// One warp per 32 x 32 tile of a task, kTaskWarps tiles per CTA.
constexpr int kTaskWarps = 4;

template <class T>
__global__ void __launch_bounds__(32 * kTaskWarps) k_tasks(const Task* __restrict__ tasks,
                                                           const int64_t* __restrict__ tstart,
                                                           int ntasks, int64_t ntiles,
                                                           T* __restrict__ F, T* __restrict__ SA,
                                                           const int* __restrict__ rp,
                                                           const int* __restrict__ ci,
                                                           const double* __restrict__ va,
                                                           const int* __restrict__ dofs,
                                                           const double* __restrict__ scale) {
  __shared__ T sm[kTaskWarps][kTaskTile][kTaskTile + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t tile = ((int64_t)blockIdx.x + (int64_t)blockIdx.y * gridDim.x) * kTaskWarps + w;
  if (tile >= ntiles) return;
  int t = 0;
  if (lane == 0) {
    int lo = 0, hi = ntasks - 1;   // last t with tstart[t] <= tile
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tstart[mid] <= tile) lo = mid;
      else hi = mid - 1;
    }
    t = lo;
  }
  t = __shfl_sync(0xffffffffu, t, 0);
  const Task Tk = tasks[t];
  const int64_t local = tile - tstart[t];
  const int tr = (Tk.rows + kTaskTile - 1) / kTaskTile;
  const int i0 = (int)(local % tr) * kTaskTile;
  const int j0 = (int)(local / tr) * kTaskTile;
  if (Tk.lower && i0 + kTaskTile - 1 < j0) return;
  T* dst = (Tk.dst_arena == AR_FRONT ? F : SA) + Tk.dst_off;
  const T* src = (Tk.src_arena == AR_FRONT ? F : SA) + Tk.src_off;
  const int rows = min(kTaskTile, Tk.rows - i0), cols = min(kTaskTile, Tk.cols - j0);
  T(*tb)[kTaskTile + 1] = sm[w];
  const int i = i0 + lane;   // this lane's row of the tile in the column-major writes
  if (Tk.kind == TK_COPY && Tk.trans) {
    // dst(i, j) = src[j + i*ld]: read src rows with lanes along j, write dst
    // columns with lanes along i, through the warp's shared-memory tile
    for (int ii = 0; ii < rows; ii++)
      if (lane < cols) tb[ii][lane] = src[(j0 + lane) + (int64_t)(i0 + ii) * Tk.src_ld];
    __syncwarp();
    if (lane < rows)
      for (int jj = 0; jj < cols; jj++)
        if (!Tk.lower || i >= j0 + jj) dst[i + (int64_t)(j0 + jj) * Tk.dst_ld] = tb[lane][jj];
    return;
  }
  if (Tk.kind == TK_SPARSE) {
    // values of this task's matrix: src_off is the element offset of its CSR
    // values (0 but for the serving loop's batches of several matrices)
    va += Tk.src_off;
    // A(r, c) for the tile (Sparse::operator(), src/LinAlg/sparse.cpp:80-92):
    // lane j holds column DOF c_j; every row's CSR entries are read once (all
    // lanes load the same addresses) and matched against the lanes' columns
    const int cj = lane < cols ? dofs[Tk.col_dof + j0 + lane] : -1;
    const double sc = (scale && lane < cols) ? scale[cj] : 1.0;
    // row DOFs, row extents and row scales of the tile, one per lane
    const int rl = lane < rows ? dofs[Tk.row_dof + i0 + lane] : 0;
    const int pl0 = lane < rows ? rp[rl] : 0, pl1 = lane < rows ? rp[rl + 1] : 0;
    const double srl = (scale && lane < rows) ? scale[rl] : 1.0;
#pragma unroll 4
    for (int ii = 0; ii < rows; ii++) {
      const int p0 = __shfl_sync(0xffffffffu, pl0, ii), p1 = __shfl_sync(0xffffffffu, pl1, ii);
      const double sr = __shfl_sync(0xffffffffu, srl, ii);
      double v = 0.0;
#pragma unroll
      for (int q = 0; q < 8; q++)   // stencil rows are short: independent loads
        if (p0 + q < p1 && ci[p0 + q] == cj) v = va[p0 + q];
      for (int p = p0 + 8; p < p1; p++)
        if (ci[p] == cj) v = va[p];
      if (scale) v = v * sr * sc;   // symmetric diagonal scaling
      tb[ii][lane] = (T)v;
    }
    __syncwarp();
    if (lane < rows)
      for (int jj = 0; jj < cols; jj++)
        if (!Tk.lower || i >= j0 + jj) dst[i + (int64_t)(j0 + jj) * Tk.dst_ld] = tb[lane][jj];
    return;
  }
  if (lane >= rows) return;
  for (int jj = 0; jj < cols; jj++) {
    const int j = j0 + jj;
    if (Tk.lower && i < j) continue;
    T* d = dst + i + (int64_t)j * Tk.dst_ld;
    if (Tk.kind == TK_ZERO) *d = T(0);
    else if (Tk.kind == TK_COPY) *d = src[i + (int64_t)j * Tk.src_ld];
    else *d = *d + src[i + (int64_t)j * Tk.src_ld];   // TK_ADD
  }
}

// ---------------------------------------------------------------------------
// Partial Cholesky building blocks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void report(DevError* err, int code, int front, int col) {
  if (atomicCAS(&err->code, 0, code) == 0) {
    err->front = front;
    err->col = col;
  }
}

constexpr unsigned kFull = 0xffffffffu;

// Cholesky of a kb x kb (kb <= 32) SPD block held one row per lane (row[t] is
// element (lane, t), lower triangle).  Each pivot is scaled by 1/sqrt(d) from
// rsqrt(d), so the column scaling is a multiply; lane j keeps 1/L(j,j) in
// `inv`.  Returns the first failing column or -1.
__device__ __forceinline__ int warp_potrf32(double (&row)[kPanel], int lane, int kb, double& inv) {
  int bad = -1;
  inv = 1.0;
#pragma unroll
  for (int j = 0; j < kPanel; j++) {
    if (j < kb) {
      double djj = __shfl_sync(kFull, row[j], j);
      if (!(djj > 0.0)) {               // non-positive or NaN pivot: not SPD
        if (bad < 0) bad = j;
        djj = 1.0;
      }
      const double r = rsqrt(djj);
      if (lane == j) {
        row[j] = djj * r;
        inv = r;
      } else if (lane > j) {
        row[j] = row[j] * r;
      }
#pragma unroll
      for (int l = j + 1; l < kPanel; l++) {
        const double llj = __shfl_sync(kFull, row[j], l);
        if (lane >= l && l < kb) row[l] -= row[j] * llj;
      }
    }
  }
  return bad;
}

// Load the kb x kb diagonal block at (k, k) of A into one row per lane, factor
// it, write it back to A and to Ds / Dinv (shared).  Called by one full warp.
__device__ __forceinline__ void warp_factor_diag(double* A, int64_t ld, int k, int kb,
                                                 double (*Ds)[kPanel + 1], double* Dinv,
                                                 DevError* err, int f) {
  const int lane = threadIdx.x & 31;
  double row[kPanel];
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    row[t] = (lane < kb && t < kb && t <= lane) ? A[(k + lane) + (int64_t)(k + t) * ld] : 0.0;
  double inv;
  const int bad = warp_potrf32(row, lane, kb, inv);
  if (bad >= 0 && lane == 0) report(err, 1, f, k + bad);
#pragma unroll
  for (int t = 0; t < kPanel; t++) {
    if (lane < kb && t < kb && t <= lane) A[(k + lane) + (int64_t)(k + t) * ld] = row[t];
    Ds[lane][t] = row[t];
  }
  Dinv[lane] = inv;
}

// Left-looking Cholesky of the kb x kb diagonal block at (k, k) of A by one
// warp, followed by the explicit inverse of the factor.  Lane i keeps row i in
// registers; column j is finished with a dot product against row j (published
// in Ls) and a reciprocal square root, so the dependent chain per column is
// short.  On exit A and Ls hold L, Li holds L^{-1} (lower, stride kLi) and
// Dinv the reciprocals of the diagonal.  Called by one full warp.
constexpr int kLi = 36;
__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }

template <class T>
__device__ void warp_factor_inv(T* A, int64_t ld, int k, int kb, T (*Ls)[kPanel + 1],
                                T* Li, T* Dinv, DevError* err, int f) {
  const int lane = threadIdx.x & 31;
  T row[kPanel];
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    row[t] = (lane < kb && t < kb && t <= lane) ? A[(k + lane) + (int64_t)(k + t) * ld] : T(0);
  int bad = -1;
#pragma unroll
  for (int j = 0; j < kPanel; j++) {
    if (j < kb) {
      T s0 = row[j], s1 = T(0), s2 = T(0), s3 = T(0);
#pragma unroll
      for (int t = 0; t < j; t++) {
        const T l = Ls[j][t];
        if ((t & 3) == 0) s0 -= row[t] * l;
        else if ((t & 3) == 1) s1 -= row[t] * l;
        else if ((t & 3) == 2) s2 -= row[t] * l;
        else s3 -= row[t] * l;
      }
      const T sv = (s0 + s1) + (s2 + s3);
      T piv = __shfl_sync(kFull, sv, j);
      if (!(piv > T(0))) {                // non-positive or NaN pivot: not SPD
        if (bad < 0) bad = j;
        piv = T(1);
      }
      const T r = rsq(piv);
      row[j] = lane == j ? piv * r : (lane > j ? sv * r : T(0));
      if (lane >= j && lane < kb) Ls[lane][j] = row[j];
      if (lane == j) Dinv[j] = r;
      __syncwarp();
    }
  }
  if (bad >= 0 && lane == 0) report(err, 1, f, k + bad);
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    if (lane < kb && t < kb && t <= lane) A[(k + lane) + (int64_t)(k + t) * ld] = row[t];
  // inverse: lane c computes column c, x_i = -(sum_{c<=t<i} L(i,t) x_t) / L(i,i)
  T x[kPanel];
#pragma unroll
  for (int i = 0; i < kPanel; i++) {
    T v = T(0);
    if (i < kb) {
      T s0 = T(0), s1 = T(0), s2 = T(0), s3 = T(0);
#pragma unroll
      for (int t = 0; t < i; t++) {
        const T l = Ls[i][t];
        const T xt = t >= lane ? x[t] : T(0);
        if ((t & 3) == 0) s0 += l * xt;
        else if ((t & 3) == 1) s1 += l * xt;
        else if ((t & 3) == 2) s2 += l * xt;
        else s3 += l * xt;
      }
      const T di = Dinv[i];
      v = i == lane ? di : (i > lane ? -((s0 + s1) + (s2 + s3)) * di : T(0));
    }
    x[i] = v;
    Li[i * kLi + lane] = v;
  }
  __syncwarp();
}

// One FP64 tensor-core MMA: D(8x8) += A(8x4) B(4x8).  Fragments: a = A(lane/4,
// lane%4), b = B(lane%4, lane/4), c/d = C(lane/4, 2*(lane%4) + {0,1}).
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int kPS = 36;   // shared-memory row stride (doubles) of a staged panel

// acc(32x32) += X[I0:I0+32, 0:kk] * Y[J0:J0+32, 0:kk]^T for row-major operands
// in shared memory (strides sx, sy; rows padded with zeros to the tile edge).
// Lane (rr = lane/4, cc = lane%4) owns rows I0 + 8a + rr and columns
// J0 + 8b + 2cc + q of the tile: the FP64 tensor-core (m8n8k4) accumulator
// layout, which the FP32 version reproduces with CUDA-core FMAs.
__device__ __forceinline__ void warp_gemm_nt_acc(const double* X, int sx, int I0, const double* Y,
                                                 int sy, int J0, int kk, int lane,
                                                 double (&acc)[4][4][2]) {
  const int rr = lane >> 2, cc = lane & 3;
  for (int k = 0; k < kk; k += 4) {
    double fa[4], fb[4];
#pragma unroll
    for (int a = 0; a < 4; a++) fa[a] = X[(I0 + 8 * a + rr) * sx + k + cc];
#pragma unroll
    for (int b = 0; b < 4; b++) fb[b] = Y[(J0 + 8 * b + rr) * sy + k + cc];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) dmma(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
  }
}

__device__ __forceinline__ void warp_gemm_nt_acc(const float* X, int sx, int I0, const float* Y,
                                                 int sy, int J0, int kk, int lane,
                                                 float (&acc)[4][4][2]) {
  const int rr = lane >> 2, cc = lane & 3;
  for (int k = 0; k < kk; k++) {
    float fa[4], fb[4][2];
#pragma unroll
    for (int a = 0; a < 4; a++) fa[a] = X[(I0 + 8 * a + rr) * sx + k];
#pragma unroll
    for (int b = 0; b < 4; b++) {
      fb[b][0] = Y[(J0 + 8 * b + 2 * cc) * sy + k];
      fb[b][1] = Y[(J0 + 8 * b + 2 * cc + 1) * sy + k];
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) {
        acc[a][b][0] = fmaf(fa[a], fb[b][0], acc[a][b][0]);
        acc[a][b][1] = fmaf(fa[a], fb[b][1], acc[a][b][1]);
      }
  }
}

template <class T>
__device__ __forceinline__ void acc_zero(T (&acc)[4][4][2]) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = T(0);
}

template <class T>
__device__ __forceinline__ void warp_gemm_nt(const T* X, int sx, int I0, const T* Y, int sy, int J0,
                                             int kk, int lane, T (&acc)[4][4][2]) {
  acc_zero(acc);
  warp_gemm_nt_acc(X, sx, I0, Y, sy, J0, kk, lane, acc);
}

template <class T>
__device__ __forceinline__ void warp_syrk_tile(const T* P, int I0, int J0, int kk, int lane,
                                               T (&acc)[4][4][2]) {
  warp_gemm_nt(P, kPS, I0, P, kPS, J0, kk, lane, acc);
}

// Panel triangular solve of the 32-row block R0 of P in place with the explicit
// inverse: P(R0 block) <- P(R0 block) Li^T; rows < M are also written to A at
// (r0 + row, k + col), cols < kb.
template <class T>
__device__ __forceinline__ void warp_trsm_block(T* P, int R0, const T* Li, int kb, T* A, int64_t ld,
                                                int r0, int k, int M, int lane) {
  T acc[4][4][2];
  warp_gemm_nt(P, kPS, R0, Li, kLi, 0, (kb + 3) & ~3, lane, acc);
  __syncwarp();
  const int rr = lane >> 2, cc = lane & 3;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int row = R0 + 8 * a + rr, col = 8 * b + 2 * cc + q;
        P[row * kPS + col] = acc[a][b][q];
        if (row < M && col < kb) A[(r0 + row) + (int64_t)(k + col) * ld] = acc[a][b][q];
      }
}

// C(r0 + i, r0 + j) -= acc for the tile at (I0, J0); lower triangle and i, j < M.
template <class T>
__device__ __forceinline__ void warp_tile_sub(T* A, int64_t ld, int r0, int M, int I0, int J0,
                                              int lane, const T (&acc)[4][4][2]) {
  const int rr = lane >> 2, cc = lane & 3;
  // all loads first, then all stores, so the accesses overlap
  T cur[4][4][2];
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int j = J0 + 8 * b + 2 * cc + q;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int i = I0 + 8 * a + rr;
        cur[a][b][q] = (i < M && j < M && i >= j) ? A[(r0 + i) + (int64_t)(r0 + j) * ld] : T(0);
      }
    }
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int j = J0 + 8 * b + 2 * cc + q;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int i = I0 + 8 * a + rr;
        if (i < M && j < M && i >= j) A[(r0 + i) + (int64_t)(r0 + j) * ld] = cur[a][b][q] - acc[a][b][q];
      }
    }
}

__device__ __forceinline__ void tri_index(int t, int& I, int& J) {
  I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while (I * (I + 1) / 2 > t) I--;
  while ((I + 1) * (I + 2) / 2 <= t) I++;
  J = t - I * (I + 1) / 2;
}

// Triangular solve of one row against the factored diagonal block:
// x(0:kb) <- x L^{-T}, with the reciprocals of the diagonal in Dinv.
__device__ __forceinline__ void row_trsm(double (&x)[kPanel], const double (*L)[kPanel + 1],
                                         const double* Dinv, int kb) {
#pragma unroll
  for (int j = 0; j < kPanel; j++) {
    if (j < kb) {
      double s = x[j];
#pragma unroll
      for (int t = 0; t < j; t++) s -= x[t] * L[j][t];
      x[j] = s * Dinv[j];
    }
  }
}

// ---------------------------------------------------------------------------
// Fused partial factorization, one CTA per front (fronts up to kSmallMaxN).
// The panel of each step is staged in shared memory for the tensor-core update.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256, 2) k_front_small(const int* __restrict__ flist,
                                                     const FrontDev* __restrict__ fr,
                                                     T* __restrict__ F, DevError* err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Psm = reinterpret_cast<T*>(smraw);
  __shared__ T Ls[kPanel][kPanel + 1];
  __shared__ T Li[kPanel * kLi];
  __shared__ T Dinv[kPanel];
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  T* A = F + d.off;
  const int64_t ld = d.ld;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (warp == 0) warp_factor_inv(A, ld, 0, min(kPanel, d.n), Ls, Li, Dinv, err, f);
  for (int k = 0; k < d.n; k += kPanel) {
    const int kb = min(kPanel, d.n - k);
    const int r0 = k + kb;
    const int M = d.N - r0;
    const int Mp = (M + 31) & ~31;
    // stage the panel rows below the diagonal block (zero padded)
    for (int idx = tid; idx < Mp * kPanel; idx += blockDim.x) {
      const int rr = idx % Mp, t = idx / Mp;
      Psm[rr * kPS + t] = (rr < M && t < kb) ? A[(r0 + rr) + (int64_t)(k + t) * ld] : T(0);
    }
    __syncthreads();
    for (int R0 = warp * 32; R0 < Mp; R0 += 256) warp_trsm_block(Psm, R0, Li, kb, A, ld, r0, k, M, lane);
    __syncthreads();
    const int TT = Mp >> 5;
    const int ntile = TT * (TT + 1) / 2;
    const int kk = (kb + 3) & ~3;
    if (warp == 0) {
      // lookahead: tile (0, 0) holds the next diagonal block; update it, then
      // factor it while the other warps finish the trailing update
      if (ntile > 0) {
        T acc[4][4][2];
        warp_syrk_tile(Psm, 0, 0, kk, lane, acc);
        warp_tile_sub(A, ld, r0, M, 0, 0, lane, acc);
      }
      __syncwarp();
      if (r0 < d.n) warp_factor_inv(A, ld, r0, min(kPanel, d.n - r0), Ls, Li, Dinv, err, f);
    } else {
      for (int t = warp; t < ntile; t += 7) {   // warps 1..7 take tiles 1, 2, ...
        int I, J;
        tri_index(t, I, J);
        T acc[4][4][2];
        warp_syrk_tile(Psm, I * 32, J * 32, kk, lane, acc);
        warp_tile_sub(A, ld, r0, M, I * 32, J * 32, lane, acc);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Stepped path for large fronts: one launch per kernel per panel step, all
// fronts of the level in each launch.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32) k_potrf(const int* __restrict__ flist,
                                              const FrontDev* __restrict__ fr,
                                              double* __restrict__ F, int k, DevError* err) {
  __shared__ double Ds[kPanel][kPanel + 1];
  __shared__ double Dinv[kPanel];
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  if (k >= d.n) return;
  warp_factor_diag(F + d.off, d.ld, k, min(kPanel, d.n - k), Ds, Dinv, err, f);
}

// Rows below the diagonal block: X = A(r, k:k+kb) L_kk^{-T}.
__global__ void __launch_bounds__(128) k_trsm(const int* __restrict__ flist,
                                              const FrontDev* __restrict__ fr,
                                              double* __restrict__ F, int k) {
  const int f = flist[blockIdx.y];
  const FrontDev d = fr[f];
  if (k >= d.n) return;
  const int kb = min(kPanel, d.n - k);
  __shared__ double L[kPanel][kPanel + 1];
  __shared__ double Linv[kPanel];
  double* A = F + d.off;
  for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
    int i = idx % kb, j = idx / kb;
    if (i >= j) L[i][j] = A[(k + i) + (int64_t)(k + j) * d.ld];
  }
  __syncthreads();
  if (threadIdx.x < kb) Linv[threadIdx.x] = 1.0 / L[threadIdx.x][threadIdx.x];
  __syncthreads();
  const int r = k + kb + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.N) return;
  double x[kPanel];
#pragma unroll
  for (int t = 0; t < kPanel; t++) x[t] = t < kb ? A[r + (int64_t)(k + t) * d.ld] : 0.0;
  row_trsm(x, L, Linv, kb);
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    if (t < kb) A[r + (int64_t)(k + t) * d.ld] = x[t];
}

// Trailing update C(r, c) -= sum_t X(r, t) X(c, t), r >= c, over [k+kb, N)^2,
// 64 x 64 tiles per CTA (four warps of 32 x 32) on the FP64 tensor cores.
constexpr int UT = 64;
__global__ void __launch_bounds__(128) k_syrk(const int* __restrict__ flist,
                                              const FrontDev* __restrict__ fr,
                                              double* __restrict__ F, int k) {
  const int f = flist[blockIdx.y];
  const FrontDev d = fr[f];
  if (k >= d.n) return;
  const int kb = min(kPanel, d.n - k);
  const int r0 = k + kb;
  const int M = d.N - r0;
  if (M <= 0) return;
  const int T = (M + UT - 1) / UT;
  if ((int)blockIdx.x >= T * (T + 1) / 2) return;
  int I, J;
  tri_index(blockIdx.x, I, J);
  __shared__ double Xa[UT * kPS];
  __shared__ double Xb[UT * kPS];
  double* A = F + d.off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int idx = tid; idx < UT * kPanel; idx += blockDim.x) {
    const int i = idx % UT, t = idx / UT;
    const int ra = r0 + I * UT + i, rb = r0 + J * UT + i;
    const bool ok = t < kb;
    Xa[i * kPS + t] = (ok && ra < d.N) ? A[ra + (int64_t)(k + t) * d.ld] : 0.0;
    Xb[i * kPS + t] = (ok && rb < d.N) ? A[rb + (int64_t)(k + t) * d.ld] : 0.0;
  }
  __syncthreads();
  const int wi = warp >> 1, wj = warp & 1;
  if (I == J && wi < wj) return;             // strictly upper quarter of a diagonal tile
  double acc[4][4][2];
  const int kk = (kb + 3) & ~3;
  {  // tile rows from Xa, tile columns from Xb
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int rr = lane >> 2, cc = lane & 3;
    for (int t = 0; t < kk; t += 4) {
      double fa[4], fb[4];
#pragma unroll
      for (int a = 0; a < 4; a++) fa[a] = Xa[(wi * 32 + 8 * a + rr) * kPS + t + cc];
#pragma unroll
      for (int b = 0; b < 4; b++) fb[b] = Xb[(wj * 32 + 8 * b + rr) * kPS + t + cc];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) dmma(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
    }
  }
  warp_tile_sub(A, d.ld, r0, M, I * UT + wi * 32, J * UT + wj * 32, lane, acc);
}

// ---------------------------------------------------------------------------
// Large fronts: one cooperative persistent launch per level.  Two-level
// blocking: outer panels of `outer` columns (kOuter = 512 unless the caller
// asks for narrower ones); inside each, 32-column steps
//   A  triangular solve of the rows below the diagonal block (every work item
//      factors the 32 x 32 diagonal block itself, from the not yet overwritten
//      values, so no extra phase is needed),
//   B  the diagonal block is written back and the outer panel's remaining
//      columns are updated with the 32 new columns,
// and after the outer panel
//   C  the trailing matrix is updated with the whole outer panel.
// Phases are separated by grid-wide barriers; work items (row blocks, 64 x 64
// tiles) of all fronts of the level are spread over all CTAs.
// ---------------------------------------------------------------------------
constexpr int kOuter = 512;
constexpr int kCT = 128;           // threads per CTA of the cooperative kernel
constexpr int kMaxCoopFronts = 8192;

// C(tile) -= X(rows) X(cols)^T over columns [k0, k1) of the front, 64 x 64 tile
// at rows [ri, ri+64), cols [ci, ci+64); rows < N, cols < cmax, row >= col.
template <class T>
__device__ void coop_tile_update(T* A, int64_t ld, int N, int cmax, int ri, int ci, int k0, int k1,
                                 T* Xa, T* Xb) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wi = warp >> 1, wj = warp & 1;
  T acc[4][4][2];
  acc_zero(acc);
  const bool diag = (ri == ci);
  const bool live = !(diag && wi < wj);
  for (int kc = k0; kc < k1; kc += kPanel) {
    const int kb = min(kPanel, k1 - kc);
    __syncthreads();
    for (int idx = tid; idx < 64 * kPanel; idx += kCT) {
      const int i = idx % 64, t = idx / 64;
      const bool ok = t < kb;
      const int ra = ri + i, rb = ci + i;
      Xa[i * kPS + t] = (ok && ra < N) ? A[ra + (int64_t)(kc + t) * ld] : T(0);
      Xb[i * kPS + t] = (ok && rb < N) ? A[rb + (int64_t)(kc + t) * ld] : T(0);
    }
    __syncthreads();
    if (live) warp_gemm_nt_acc(Xa, kPS, wi * 32, Xb, kPS, wj * 32, (kb + 3) & ~3, lane, acc);
  }
  if (!live) return;
  const int rr = lane >> 2, cc = lane & 3;
  // all loads first, then all stores, so the accesses overlap
  T cur[4][4][2];
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int c = ci + wj * 32 + 8 * b + 2 * cc + q;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int r = ri + wi * 32 + 8 * a + rr;
        cur[a][b][q] = (r < N && c < cmax && r >= c) ? A[r + (int64_t)c * ld] : T(0);
      }
    }
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int c = ci + wj * 32 + 8 * b + 2 * cc + q;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int r = ri + wi * 32 + 8 * a + rr;
        if (r < N && c < cmax && r >= c) A[r + (int64_t)c * ld] = cur[a][b][q] - acc[a][b][q];
      }
    }
}

// Factored diagonal blocks are handed from the CTA that completes their update
// to every work item of the next step through a per-front slot in global
// memory holding the inverse of the factor (32 rows of stride kLi).
constexpr int kDiagSlot = kPanel * kLi;

// Warp 0 of the calling CTA factors the diagonal block at (k, k), writes it
// back into the front and publishes it in `slot`.  Every thread must call.
template <class T>
__device__ void coop_factor_publish(T* A, int64_t ld, int k, int kb, T* slot,
                                    T (*Ls)[kPanel + 1], T* Li, T* Dinv,
                                    DevError* err, int f) {
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    warp_factor_inv(A, ld, k, kb, Ls, Li, Dinv, err, f);
    for (int i = 0; i < kPanel; i++) slot[i * kLi + lane] = Li[i * kLi + lane];
  }
}

__device__ __forceinline__ int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Per-phase work-item prefixes come from the host (coop_phase_prefix): for
// phase p, pref[p * (nf + 1) + i] is the first item of front i.  Each CTA
// copies the phase's prefix into shared memory and binary-searches it.
//
// One launch covers the outer panels [K0, K1) (K0 a multiple of outer);
// phase0 is the index of the first phase of outer panel K0 in phase_pref.  With
// trailing == 0 the last outer panel's phase C is left to the caller (the
// tensor-core trailing update of the mixed path), and the next launch factors
// and publishes its first diagonal block itself.
template <class T>
__global__ void __launch_bounds__(kCT) k_level_coop(const int* __restrict__ flist, int nf,
                                                    const FrontDev* __restrict__ fr,
                                                    T* __restrict__ F, DevError* err, int maxn,
                                                    T* __restrict__ slots,
                                                    const int* __restrict__ phase_pref, int K0,
                                                    int K1, int phase0, int trailing, int outer,
                                                    unsigned* gbar) {
  unsigned gtarget = 0;
  __shared__ T Ls[kPanel][kPanel + 1];
  __shared__ T Li[kPanel * kLi];
  __shared__ T Dinv[kPanel];
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Xa = reinterpret_cast<T*>(smraw);      // phase B / C tile operands
  T* Xb = Xa + 64 * kPS;
  T* Rows = Xa;                             // phase A: kCT = 128 staged rows
  int* pre = reinterpret_cast<int*>(Xa + 2 * 64 * kPS);
  const int tid = threadIdx.x;
  int phase = phase0;
  auto load_phase = [&]() {
    __syncthreads();
    const int* p = phase_pref + (int64_t)(phase++) * (nf + 1);
    for (int i = tid; i <= nf; i += kCT) pre[i] = p[i];
    __syncthreads();
  };
  auto find = [&](int item) {   // largest i with pre[i] <= item
    int lo = 0, hi = nf - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  };
  // the first diagonal block of every front
  for (int i = blockIdx.x; i < nf; i += gridDim.x) {
    const int f = flist[i];
    const FrontDev d = fr[f];
    if (d.n > K0)
      coop_factor_publish(F + d.off, d.ld, K0, min(kPanel, d.n - K0), slots + (int64_t)i * kDiagSlot,
                          Ls, Li, Dinv, err, f);
  }
  grid_barrier(gbar, gtarget, err);
  for (int K = K0; K < K1 && K < maxn; K += outer) {
    for (int k = K; k < K + outer && k < maxn; k += kPanel) {
      // ---- phase A: rows below the (already factored) diagonal block ----
      load_phase();
      for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
        const int i = find(item);
        const FrontDev d = fr[flist[i]];
        T* A = F + d.off;
        const int kb = min(kPanel, d.n - k);
        const T* slot = slots + (int64_t)i * kDiagSlot;
        const int rbase = k + kb + (item - pre[i]) * kCT;
        const int Mi = min(kCT, d.N - rbase);
        __syncthreads();
        for (int idx = tid; idx < kPanel * kLi; idx += kCT) Li[idx] = slot[idx];
        for (int idx = tid; idx < kCT * kPanel; idx += kCT) {
          const int rr = idx % kCT, t = idx / kCT;
          Rows[rr * kPS + t] = (rr < Mi && t < kb) ? A[(rbase + rr) + (int64_t)(k + t) * d.ld] : T(0);
        }
        __syncthreads();
        warp_trsm_block(Rows, (tid >> 5) * 32, (const T*)Li, kb, A, d.ld, rbase, k, Mi, tid & 31);
      }
      grid_barrier(gbar, gtarget, err);
      // ---- phase B: update the outer panel's remaining columns; the CTA that
      // updates the next diagonal block factors and publishes it ----
      load_phase();
      for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
        const int i = find(item);
        const int f = flist[i];
        const FrontDev d = fr[f];
        T* A = F + d.off;
        const int kb = min(kPanel, d.n - k);
        int local = item - pre[i];
        const int c0 = k + kb, cmax = min(K + outer, d.n);
        const int TI = ceil_div(d.N - c0, 64);
        int J = 0;
        while (local >= TI - J) {
          local -= TI - J;
          J++;
        }
        const int I = J + local;
        coop_tile_update(A, d.ld, d.N, cmax, c0 + I * 64, c0 + J * 64, k, k + kb, Xa, Xb);
        if (I == 0 && J == 0)
          coop_factor_publish(A, d.ld, c0, min(kPanel, d.n - c0), slots + (int64_t)i * kDiagSlot, Ls,
                              Li, Dinv, err, f);
      }
      grid_barrier(gbar, gtarget, err);
    }
    // ---- phase C: trailing update with the outer panel ----
    if (!trailing && K + outer >= K1) break;
    load_phase();
    for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
      const int i = find(item);
      const int f = flist[i];
      const FrontDev d = fr[f];
      const int k1 = min(K + outer, d.n);
      int I, J;
      tri_index(item - pre[i], I, J);
      coop_tile_update(F + d.off, d.ld, d.N, d.N, k1 + I * 64, k1 + J * 64, K, k1, Xa, Xb);
      if (I == 0 && J == 0 && k1 < d.n)
        coop_factor_publish(F + d.off, d.ld, k1, min(kPanel, d.n - k1), slots + (int64_t)i * kDiagSlot,
                            Ls, Li, Dinv, err, f);
    }
    grid_barrier(gbar, gtarget, err);
  }
}

// Trailing update of the panel-by-panel factorization (kernels_panel.cu):
// C(k1:N, k1:N) -= P P^T, P = L(k1:N, Ks:k1), k1 = min(Ks + w, n), lower
// 64 x 64 tiles of every front over a persistent grid.
template <class T>
__global__ void __launch_bounds__(kCT) k_trail_syrk(const int* __restrict__ flist, int nf,
                                                    const FrontDev* __restrict__ fr,
                                                    T* __restrict__ F, int Ks, int w) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Xa = reinterpret_cast<T*>(smraw);
  T* Xb = Xa + 64 * kPS;
  __shared__ int pre[kMaxPanelFronts + 1];
  const int tid = threadIdx.x;
  for (int i = tid; i < nf; i += kCT) {
    const FrontDev d = fr[flist[i]];
    const int k1 = min(Ks + w, d.n), t = (d.N - k1 + 63) / 64;
    pre[i + 1] = Ks < d.n && d.N > k1 ? t * (t + 1) / 2 : 0;
  }
  __syncthreads();
  if (tid == 0) {
    pre[0] = 0;
    for (int i = 0; i < nf; i++) pre[i + 1] += pre[i];
  }
  __syncthreads();
  const int total = pre[nf];
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    int lo = 0, hi = nf - 1;   // largest i with pre[i] <= item
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    const FrontDev d = fr[flist[lo]];
    const int k1 = min(Ks + w, d.n);
    int I, J;
    tri_index(item - pre[lo], I, J);
    coop_tile_update(F + d.off, d.ld, d.N, d.N, k1 + I * 64, k1 + J * 64, Ks, k1, Xa, Xb);
  }
}

// ---------------------------------------------------------------------------
// Solve / apply sweeps.  One CTA per front; W is the front's workspace (N x nrhs,
// ld N) inside a shared buffer.
// ---------------------------------------------------------------------------
constexpr int ST = 256;

// Forward solve with the front's first n columns, right-looking over 32-column
// blocks.  On exit W[0,n) = L11^{-1} b_piv and W[n,N) = -L21 W[0,n).  W is the
// front's right-hand-side block (N x nrhs, ld N) in shared or global memory.
// UNIT: L11 has a unit diagonal (the L of a pivoted LU front) and its stored
// diagonal, U's, is not read.
template <class T, int NR, bool UNIT = false>
__device__ void front_forward(const FrontDev& d, const T* __restrict__ A, T* W,
                              int nrhs) {
  __shared__ T Ls[kPanel][kPanel + 1];
  __shared__ T xs[kPanel][NR + 1];
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  for (int k = 0; k < n; k += kPanel) {
    const int kb = min(kPanel, n - k);
    for (int idx = tid; idx < kb * kb; idx += blockDim.x) {
      const int i = idx % kb, j = idx / kb;
      if (i >= j) Ls[i][j] = A[(k + i) + (int64_t)(k + j) * ld];
    }
    for (int idx = tid; idx < kb * nrhs; idx += blockDim.x) {
      const int i = idx % kb, c = idx / kb;
      xs[i][c] = W[k + i + (int64_t)c * N];
    }
    __syncthreads();
    if (warp == 0) {
      // column-oriented substitution: lane i owns row i of the block
      for (int j = 0; j < kb; j++) {
        if (!UNIT && lane == j) {
          const T djj = Ls[j][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[j][c] = xs[j][c] / djj;
        }
        __syncwarp();
        if (lane > j && lane < kb) {
          const T l = Ls[lane][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[lane][c] -= l * xs[j][c];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int idx = tid; idx < kb * nrhs; idx += blockDim.x) {
      const int i = idx % kb, c = idx / kb;
      W[k + i + (int64_t)c * N] = xs[i][c];
    }
    // rows below the block: W(r, :) -= L(r, k:k+kb) x   (thread per row, coalesced L)
    for (int r = k + kb + tid; r < N; r += blockDim.x) {
      T acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = T(0);
      const T* Lr = A + r + (int64_t)k * ld;
      if (kb == kPanel) {
        // all 32 loads issued before the FMAs: memory-level parallelism
        T l[kPanel];
#pragma unroll
        for (int t = 0; t < kPanel; t++) l[t] = Lr[(int64_t)t * ld];
#pragma unroll
        for (int t = 0; t < kPanel; t++)
#pragma unroll
          for (int c = 0; c < NR; c++) acc[c] = fma(l[t], xs[t][c], acc[c]);
      } else {
        for (int t = 0; t < kb; t++) {
          const T l = Lr[(int64_t)t * ld];
#pragma unroll
          for (int c = 0; c < NR; c++) acc[c] = fma(l, xs[t][c], acc[c]);
        }
      }
#pragma unroll
      for (int c = 0; c < NR; c++)
        if (c < nrhs) W[r + (int64_t)c * N] -= acc[c];
    }
    __syncthreads();
  }
}

// Backward solve: W[0,n) <- L11^{-T} (W[0,n) - L21^T W[n,N)).
template <class T, int NR>
__device__ void front_backward(const FrontDev& d, const T* __restrict__ A, T* W,
                               int nrhs) {
  __shared__ T Ls[kPanel][kPanel + 1];
  __shared__ T xs[kPanel][NR + 1];
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int nblk = (n + kPanel - 1) / kPanel;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int k = bk * kPanel;
    const int kb = min(kPanel, n - k);
    for (int idx = tid; idx < kb * kb; idx += blockDim.x) {
      const int i = idx % kb, j = idx / kb;
      if (i >= j) Ls[i][j] = A[(k + i) + (int64_t)(k + j) * ld];
    }
    // xs(j, c) = W(k+j, c) - sum_{r >= k+kb} L(r, k+j) W(r, c): warp per column
    for (int j = warp; j < kb; j += nw) {
      T acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = T(0);
      const T* Lc = A + (int64_t)(k + j) * ld;
      int r = k + kb + lane;
      for (; r + 96 < N; r += 128) {      // four independent loads in flight
        const T l0 = Lc[r], l1 = Lc[r + 32], l2 = Lc[r + 64], l3 = Lc[r + 96];
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) {
            const T* w = W + (int64_t)c * N + r;
            acc[c] = fma(l0, w[0], acc[c]);
            acc[c] = fma(l1, w[32], acc[c]);
            acc[c] = fma(l2, w[64], acc[c]);
            acc[c] = fma(l3, w[96], acc[c]);
          }
      }
      for (; r < N; r += 32) {
        const T l = Lc[r];
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) acc[c] = fma(l, W[r + (int64_t)c * N], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < NR; c++) {
        T v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && c < nrhs) xs[j][c] = W[k + j + (int64_t)c * N] - v;
      }
    }
    __syncthreads();
    if (warp == 0) {
      for (int j = kb - 1; j >= 0; j--) {
        if (lane == j) {
          const T djj = Ls[j][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[j][c] = xs[j][c] / djj;
        }
        __syncwarp();
        if (lane < j) {
          const T l = Ls[j][lane];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[lane][c] -= l * xs[j][c];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int idx = tid; idx < kb * nrhs; idx += blockDim.x) {
      const int i = idx % kb, c = idx / kb;
      W[k + i + (int64_t)c * N] = xs[i][c];
    }
    __syncthreads();
  }
}

// Shared-memory staging of a front's right-hand-side block when it fits.
constexpr int kSolveSmemBytes = 200 * 1024;


template <class T, int NR>
__global__ void __launch_bounds__(ST) k_solve_fwd(const int* __restrict__ flist,
                                                  const FrontDev* __restrict__ fr,
                                                  const T* __restrict__ F,
                                                  const int* __restrict__ dofs, T* X,
                                                  int64_t ldx, int nrhs, T* Wb,
                                                  const int64_t* __restrict__ woff, int use_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* smW = reinterpret_cast<T*>(smraw);
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  T* Wg = Wb + woff[f] * nrhs;
  T* W = use_smem ? smW : Wg;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = i < d.n ? X[dl[i] + (int64_t)c * ldx] : T(0);
  }
  __syncthreads();
  front_forward<T, NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    if (i < d.n) X[dl[i] + (int64_t)c * ldx] = W[idx];
    else if (use_smem) Wg[idx] = W[idx];    // boundary part for the separator gather
  }
}

template <class T, int NR>
__global__ void __launch_bounds__(ST) k_solve_bwd(const int* __restrict__ flist,
                                                  const FrontDev* __restrict__ fr,
                                                  const T* __restrict__ F,
                                                  const int* __restrict__ dofs, T* X,
                                                  int64_t ldx, int nrhs, T* Wb,
                                                  const int64_t* __restrict__ woff, int use_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* smW = reinterpret_cast<T*>(smraw);
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  T* W = use_smem ? smW : Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  front_backward<T, NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

template <class T, int NR>
__global__ void __launch_bounds__(ST) k_root_solve(int f, const FrontDev* __restrict__ fr,
                                                   const T* __restrict__ F,
                                                   const int* __restrict__ dofs, T* X,
                                                   int64_t ldx, int nrhs, T* Wb,
                                                   const int64_t* __restrict__ woff, int use_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* smW = reinterpret_cast<T*>(smraw);
  const FrontDev d = fr[f];
  T* W = use_smem ? smW : Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  front_forward<T, NR>(d, F + d.off, W, nrhs);
  front_backward<T, NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

// X(sep) = (X(sep) + W_box0(sep rows)) + W_box1(sep rows), the reference's
// per-box accumulation order (mf2d.cpp:992-1011, 1036-1047).
template <class T>
__global__ void __launch_bounds__(ST) k_sep_gather(const int* __restrict__ slist,
                                                   const SepDev* __restrict__ sp,
                                                   const int* __restrict__ dofs, T* X,
                                                   int64_t ldx, int nrhs,
                                                   const T* __restrict__ Wb,
                                                   const int64_t* __restrict__ woff,
                                                   const FrontDev* __restrict__ fr) {
  const SepDev s = sp[slist[blockIdx.x]];
  const int* dl = dofs + s.dof_off;
  const int N0 = fr[s.box0].N, N1 = fr[s.box1].N;
  const T* W0 = Wb + woff[s.box0] * nrhs;
  const T* W1 = Wb + woff[s.box1] * nrhs;
  for (int idx = threadIdx.x; idx < s.s * nrhs; idx += blockDim.x) {
    const int i = idx % s.s, c = idx / s.s;
    T* x = X + dl[i] + (int64_t)c * ldx;
    *x = (*x + W0[s.pos0 + i + (int64_t)c * N0]) + W1[s.pos1 + i + (int64_t)c * N1];
  }
}

// Apply, upward part: t = L11^T b_piv + L21^T b_bd ; b_piv = L11 t ; T(piv) = t.
template <class T>
__device__ void front_apply_up(const FrontDev& d, const T* __restrict__ A, T* W,
                               T* Tt, int nrhs) {
  // W holds [b_piv; b_bd] (N x nrhs); Tt receives t (n x nrhs, ld n).
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int jc = warp; jc < n * nrhs; jc += nw) {
    const int j = jc % n, c = jc / n;
    const T* w = W + (int64_t)c * N;
    T s = T(0);
    for (int r = j + lane; r < N; r += 32) s += A[r + (int64_t)j * ld] * w[r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) Tt[j + (int64_t)c * n] = s;
  }
  __syncthreads();
  for (int idx = tid; idx < n * nrhs; idx += blockDim.x) {
    const int r = idx % n, c = idx / n;
    const T* t = Tt + (int64_t)c * n;
    T s = T(0);
    for (int j = 0; j <= r; j++) s += A[r + (int64_t)j * ld] * t[j];
    W[r + (int64_t)c * N] = s;
  }
  __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(ST) k_apply_up(const int* __restrict__ flist,
                                                 const FrontDev* __restrict__ fr,
                                                 const T* __restrict__ F,
                                                 const int* __restrict__ dofs, T* X,
                                                 int64_t ldx, int nrhs, T* Wb,
                                                 const int64_t* __restrict__ woff, T* Tb) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  T* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  T* Tt = W + (int64_t)d.N * nrhs;  // second half of the front's workspace
  front_apply_up(d, F + d.off, W, Tt, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
    Tb[dl[i] + (int64_t)c * ldx] = Tt[i + (int64_t)c * d.n];
  }
}

// Apply, downward part: W[n,N) = L21 t (t read from T by DOF).
template <class T>
__global__ void __launch_bounds__(ST) k_apply_down(const int* __restrict__ flist,
                                                   const FrontDev* __restrict__ fr,
                                                   const T* __restrict__ F,
                                                   const int* __restrict__ dofs, int64_t ldx,
                                                   int nrhs, T* Wb,
                                                   const int64_t* __restrict__ woff,
                                                   const T* __restrict__ Tb) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  T* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  const T* A = F + d.off;
  T* Tt = W + (int64_t)d.N * nrhs;
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    Tt[i + (int64_t)c * d.n] = Tb[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < d.m * nrhs; idx += blockDim.x) {
    const int r = d.n + idx % d.m, c = idx / d.m;
    const T* t = Tt + (int64_t)c * d.n;
    T s = T(0);
    for (int j = 0; j < d.n; j++) s += A[r + (int64_t)j * d.ld] * t[j];
    W[r + (int64_t)c * d.N] = s;
  }
}

template <class T>
__global__ void __launch_bounds__(ST) k_root_apply(int f, const FrontDev* __restrict__ fr,
                                                   const T* __restrict__ F,
                                                   const int* __restrict__ dofs, T* X,
                                                   int64_t ldx, int nrhs, T* Wb,
                                                   const int64_t* __restrict__ woff) {
  const FrontDev d = fr[f];
  T* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  T* Tt = W + (int64_t)d.N * nrhs;
  front_apply_up(d, F + d.off, W, Tt, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

// ---------------------------------------------------------------------------
// Sweeps of pivoted LU fronts (nonsymmetric problems, FP64; factors from
// kernels_lu.cu: P A22 = L11 U11, L21 = A12 U11^{-1}, U12 = L11^{-1} P A21).
// The reference's upward step b_sk -= XL b_rd, b_rd <- A22^{-1} b_rd and
// downward step b_rd -= XR b_sk (src/DE/mf2d.cpp:976-1054) become
//   forward:  y = L11^{-1} P b_piv (kept as the pivot part), W[n,N) = -L21 y
//   backward: x_piv = U11^{-1} (y - U12 x_bd)
// since XL = L21 L11^{-1} P and XR = U11^{-1} U12.
// ---------------------------------------------------------------------------

// Backward solve: W[0,n) <- U11^{-1} (W[0,n) - U12 W[n,N)), upward over
// 32-row blocks; U(k block, right of it) is read a column at a time (lanes
// along the block's rows), warps splitting the columns.
template <int NR>
__device__ void front_backward_lu(const FrontDev& d, const double* __restrict__ A, double* W,
                                  int nrhs) {
  __shared__ double Us[kPanel][kPanel + 1];
  __shared__ double xs[kPanel][NR + 1];
  __shared__ double part[ST / 32][kPanel];
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int nblk = (n + kPanel - 1) / kPanel;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int k = bk * kPanel, kb = min(kPanel, n - k);
    for (int idx = tid; idx < kb * kb; idx += blockDim.x) {
      const int i = idx % kb, j = idx / kb;
      if (i <= j) Us[i][j] = A[(k + i) + (int64_t)(k + j) * ld];
    }
    double acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = 0.0;
    if (lane < kb)
      for (int r = k + kb + warp; r < N; r += nw) {
        const double u = A[(k + lane) + (int64_t)r * ld];
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) acc[c] = fma(u, W[r + (int64_t)c * N], acc[c]);
      }
#pragma unroll
    for (int c = 0; c < NR; c++) {
      if (c < nrhs) {
        part[warp][lane] = acc[c];
        __syncthreads();
        if (warp == 0 && lane < kb) {
          double s = 0.0;
          for (int w = 0; w < nw; w++) s += part[w][lane];
          xs[lane][c] = W[k + lane + (int64_t)c * N] - s;
        }
        __syncthreads();
      }
    }
    if (warp == 0) {
      for (int j = kb - 1; j >= 0; j--) {
        if (lane == j) {
          const double ujj = Us[j][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[j][c] = xs[j][c] / ujj;
        }
        __syncwarp();
        if (lane < j) {
          const double u = Us[lane][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[lane][c] -= u * xs[j][c];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    for (int idx = tid; idx < kb * nrhs; idx += blockDim.x) {
      const int i = idx % kb, c = idx / kb;
      W[k + i + (int64_t)c * N] = xs[i][c];
    }
    __syncthreads();
  }
}

template <int NR>
__global__ void __launch_bounds__(ST) k_lu_solve_fwd(const int* __restrict__ flist,
                                                     const FrontDev* __restrict__ fr,
                                                     const double* __restrict__ F,
                                                     const int* __restrict__ ipiv,
                                                     const int* __restrict__ dofs, double* X,
                                                     int64_t ldx, int nrhs, double* Wb,
                                                     const int64_t* __restrict__ woff,
                                                     int use_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* smW = reinterpret_cast<double*>(smraw);
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* Wg = Wb + woff[f] * nrhs;
  double* W = use_smem ? smW : Wg;
  const int* dl = dofs + d.dof_off;
  const int* pv = ipiv + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = i < d.n ? X[dl[i] + (int64_t)c * ldx] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x < nrhs) {   // b_piv <- P b_piv: the swaps in factorization order
    double* w = W + (int64_t)threadIdx.x * d.N;
    for (int j = 0; j < d.n; j++) {
      const int p = pv[j];
      if (p != j) {
        const double t = w[j];
        w[j] = w[p];
        w[p] = t;
      }
    }
  }
  __syncthreads();
  front_forward<double, NR, true>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    if (i < d.n) X[dl[i] + (int64_t)c * ldx] = W[idx];
    else if (use_smem) Wg[idx] = W[idx];    // boundary part for the separator gather
  }
}

template <int NR>
__global__ void __launch_bounds__(ST) k_lu_solve_bwd(const int* __restrict__ flist,
                                                     const FrontDev* __restrict__ fr,
                                                     const double* __restrict__ F,
                                                     const int* __restrict__ dofs, double* X,
                                                     int64_t ldx, int nrhs, double* Wb,
                                                     const int64_t* __restrict__ woff,
                                                     int use_smem) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* smW = reinterpret_cast<double*>(smraw);
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = use_smem ? smW : Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  front_backward_lu<NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

// Apply, upward part, of a pivoted LU front: u = U11 b_piv + U12 b_bd,
// b_piv <- P^T L11 u (= A22 t with t = b_piv + XR b_bd), T(piv) = u; the
// downward part W[n,N) = L21 u (= XL A22 t) is k_apply_down's.
__global__ void __launch_bounds__(ST) k_lu_apply_up(const int* __restrict__ flist,
                                                    const FrontDev* __restrict__ fr,
                                                    const double* __restrict__ F,
                                                    const int* __restrict__ ipiv,
                                                    const int* __restrict__ dofs, double* X,
                                                    int64_t ldx, int nrhs, double* Wb,
                                                    const int64_t* __restrict__ woff, double* Tb) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  const int* pv = ipiv + d.dof_off;
  const double* A = F + d.off;
  const int N = d.N, n = d.n, ld = d.ld;
  for (int idx = threadIdx.x; idx < N * nrhs; idx += blockDim.x) {
    const int i = idx % N, c = idx / N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  double* u = W + (int64_t)N * nrhs;   // second half of the front's workspace (n x nrhs, ld n)
  // u(j) = sum_{c >= j} U(j, c) W(c): columns in order, rows across threads
  for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
    const int j = idx % n, c = idx / n;
    const double* w = W + (int64_t)c * N;
    double s = 0.0;
    // from the warp's first row, so that a warp's loads of a column coalesce
    for (int col = j & ~31; col < N; col++)
      if (col >= j) s += A[j + (int64_t)col * ld] * w[col];
    u[j + (int64_t)c * n] = s;
  }
  __syncthreads();
  // v(r) = u(r) + sum_{j < r} L(r, j) u(j)
  for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
    const int r = idx % n, c = idx / n;
    const double* uc = u + (int64_t)c * n;
    double s = uc[r];
    for (int j = 0; j < r; j++) s += A[r + (int64_t)j * ld] * uc[j];
    W[r + (int64_t)c * N] = s;
  }
  __syncthreads();
  if (threadIdx.x < nrhs) {   // P^T: the swaps undone in reverse order
    double* w = W + (int64_t)threadIdx.x * N;
    for (int j = n - 1; j >= 0; j--) {
      const int p = pv[j];
      if (p != j) {
        const double t = w[j];
        w[j] = w[p];
        w[p] = t;
      }
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
    const int i = idx % n, c = idx / n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * N];
    Tb[dl[i] + (int64_t)c * ldx] = u[i + (int64_t)c * n];
  }
}

}  // namespace

template <class T>
void launch_tasks(const Task* tasks, const int64_t* tstart, int ntasks, int64_t ntiles, T* fronts,
                  T* seps, const int* rp, const int* ci, const double* va, const int* dofs,
                  const double* scale, cudaStream_t st) {
  if (ntasks <= 0 || ntiles <= 0) return;
  const int64_t blocks = (ntiles + kTaskWarps - 1) / kTaskWarps;
  const int64_t gx = blocks < 65535 * 32 ? blocks : 65535 * 32;
  const int64_t gy = (blocks + gx - 1) / gx;
  k_tasks<T><<<dim3((unsigned)gx, (unsigned)gy), 32 * kTaskWarps, 0, st>>>(
      tasks, tstart, ntasks, ntiles, fronts, seps, rp, ci, va, dofs, scale);
  g_launches++;
}

void launch_potrf(const int* flist, int nf, const FrontDev* fr, double* F, int k, DevError* err,
                  cudaStream_t st) {
  if (nf <= 0) return;
  k_potrf<<<nf, 32, 0, st>>>(flist, fr, F, k, err);
  g_launches++;
}
void launch_trsm(const int* flist, int nf, const FrontDev* fr, double* F, int k, int max_rows,
                 cudaStream_t st) {
  const int rows = max_rows - k - 1;
  if (nf <= 0 || rows <= 0) return;
  k_trsm<<<dim3((rows + 127) / 128, nf), 128, 0, st>>>(flist, fr, F, k);
  g_launches++;
}
void launch_syrk(const int* flist, int nf, const FrontDev* fr, double* F, int k, int max_rows,
                 cudaStream_t st) {
  const int rows = max_rows - k - 1;
  if (nf <= 0 || rows <= 0) return;
  const int T = (rows + UT - 1) / UT;
  k_syrk<<<dim3(T * (T + 1) / 2, nf), 128, 0, st>>>(flist, fr, F, k);
  g_launches++;
}

long long launches_total() { return g_launches.load(); }

bool small_front_fits(int maxN, int elem_bytes) {
  // the staged panel (maxN x kPS) plus static shared memory must fit in 227 KB
  return (size_t)((maxN + 31) & ~31) * kPS * elem_bytes <= 200 * 1024;
}

bool coop_fits(int nf) { return nf <= kMaxCoopFronts; }
size_t coop_slot_elems() { return (size_t)kMaxCoopFronts * kDiagSlot; }

// Work items per phase of k_level_coop for fronts (n_i, N_i), in the kernel's
// phase order: for each outer panel K, for each 32-column step k, phases A and
// B; then phase C.  Returns the per-phase prefixes (nf + 1 ints each).
std::vector<int> coop_phase_prefix(const std::vector<int>& n, const std::vector<int>& N, int maxn,
                                   int outer) {
  if (outer <= 0) outer = kOuter;
  const int nf = (int)n.size();
  std::vector<int> out;
  auto cdiv = [](int a, int b) { return (a + b - 1) / b; };
  auto push = [&](auto count) {
    int acc = 0;
    out.push_back(0);
    for (int i = 0; i < nf; i++) {
      acc += count(i);
      out.push_back(acc);
    }
  };
  for (int K = 0; K < maxn; K += outer) {
    for (int k = K; k < K + outer && k < maxn; k += kPanel) {
      push([&](int i) { return k < n[i] ? cdiv(N[i] - k - std::min(kPanel, n[i] - k), kCT) : 0; });
      push([&](int i) {
        if (k >= n[i]) return 0;
        const int kb = std::min(kPanel, n[i] - k), c0 = k + kb, cmax = std::min(K + outer, n[i]);
        if (cmax <= c0) return 0;
        const int TI = cdiv(N[i] - c0, 64), TJ = cdiv(cmax - c0, 64);
        int c = 0;
        for (int J = 0; J < TJ; J++) c += TI - J;
        return c;
      });
    }
    push([&](int i) {
      const int k1 = std::min(K + outer, n[i]);
      if (K >= n[i] || N[i] <= k1) return 0;
      const int T = cdiv(N[i] - k1, 64);
      return T * (T + 1) / 2;
    });
  }
  return out;
}

int coop_outer() { return kOuter; }

int coop_phases(int K, int maxn, int outer) {
  if (outer <= 0) outer = kOuter;
  return 2 * ((std::min(outer, maxn - K) + kPanel - 1) / kPanel) + 1;
}

template <class T>
cudaError_t launch_level_coop(const int* flist, int nf, int maxn, const FrontDev* fr, T* F,
                              DevError* err, T* slots, const int* phase_pref, unsigned* gbar,
                              cudaStream_t st, int K0, int K1, int phase0, int trailing,
                              int max_items, int outer) {
  if (nf <= 0) return cudaSuccess;
  if (outer <= 0) outer = kOuter;
  if (outer % kPanel || K0 % outer) return cudaErrorInvalidValue;
  cudaError_t me = cudaMemsetAsync(gbar, 0, sizeof(unsigned), st);
  if (me != cudaSuccess) return me;
  if (K1 < 0) K1 = maxn;
  const size_t sm = 2 * 64 * kPS * sizeof(T) + (size_t)(kMaxCoopFronts + 1) * sizeof(int);
  // co-resident CTAs of this instantiation (thread-safe one-time set-up: the
  // serving loop launches from several host threads)
  static const int grid = [sm]() {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_level_coop<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_level_coop<T>, kCT, sm);
    return sms * (per > 0 ? per : 1);
  }();
  void* args[] = {(void*)&flist, (void*)&nf,    (void*)&fr,         (void*)&F,
                  (void*)&err,   (void*)&maxn,  (void*)&slots,      (void*)&phase_pref,
                  (void*)&K0,    (void*)&K1,    (void*)&phase0,     (void*)&trailing,
                  (void*)&outer, (void*)&gbar};
  // levels with little parallel work: one CTA per work item, at least an
  // eighth of the full grid (a grid barrier costs more the more CTAs arrive)
  int g = grid;
  if (max_items > 0) g = std::min(grid, std::max(max_items, std::max(1, grid / 8)));
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_level_coop<T>, dim3(g), dim3(kCT),
                                              args, sm, st);
  g_launches++;
  return e;
}

template <class T>
void launch_front_small(const int* flist, int nf, int maxN, const FrontDev* fr, T* F, DevError* err,
                        cudaStream_t st) {
  if (nf <= 0) return;
  const size_t sm = (size_t)((maxN + 31) & ~31) * kPS * sizeof(T);
  // the largest dynamic size any launch asks for, set once (launches from
  // several host threads must not race on the attribute)
  static const bool attr = (cudaFuncSetAttribute(k_front_small<T>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 200 * 1024),
                            true);
  (void)attr;
  k_front_small<T><<<nf, 256, sm, st>>>(flist, fr, F, err);
  g_launches++;
}

// Solve kernels are templated on a bound of the right-hand-side count and keep
// the front's right-hand-side block in dynamic shared memory when the largest
// front's fits.
namespace {
void smemFor(int maxN, int nrhs, size_t elem, size_t& sm, int& use) {
  const size_t need = (size_t)maxN * nrhs * elem;
  use = need <= (size_t)kSolveSmemBytes;
  sm = use ? need : 0;
}
}  // namespace

// Threads per CTA of the per-front sweeps: enough warps for the level's
// largest front (a thread per row below the diagonal block, a warp per column
// of the block), at least two and at most ST.  Small fronts (the leaves of a
// batch of thousands of them) then leave room for more CTAs per SM; every
// value is computed by the same operations in the same order whatever the
// block size, so results do not depend on it.
inline int sweep_threads(int maxN) { return std::min(ST, std::max(64, (maxN + 31) & ~31)); }

template <class T>
void launch_solve_fwd(const int* flist, int nf, int maxN, const FrontDev* fr, const T* F,
                      const int* dofs, T* X, int64_t ldx, int nrhs, T* W, const int64_t* woff,
                      cudaStream_t st) {
  if (nf <= 0) return;
  size_t sm;
  int use;
  smemFor(maxN, nrhs, sizeof(T), sm, use);
  const int threads = sweep_threads(maxN);
#define MFGPU_FWD(NR)                                                                          \
  do {                                                                                         \
    static const bool attr_ = (cudaFuncSetAttribute(k_solve_fwd<T, NR>,                     \
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                                    kSolveSmemBytes),                             \
                               true);                                                             \
    (void)attr_;                                                                                  \
    k_solve_fwd<T, NR><<<nf, threads, sm, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff, use);\
  } while (0)
  if (nrhs == 1) MFGPU_FWD(1);
  else if (nrhs <= 4) MFGPU_FWD(4);
  else if (nrhs <= 8) MFGPU_FWD(8);
  else MFGPU_FWD(16);
#undef MFGPU_FWD
  g_launches++;
}

template <class T>
void launch_solve_bwd(const int* flist, int nf, int maxN, const FrontDev* fr, const T* F,
                      const int* dofs, T* X, int64_t ldx, int nrhs, T* W, const int64_t* woff,
                      cudaStream_t st) {
  if (nf <= 0) return;
  size_t sm;
  int use;
  smemFor(maxN, nrhs, sizeof(T), sm, use);
  const int threads = sweep_threads(maxN);
#define MFGPU_BWD(NR)                                                                          \
  do {                                                                                         \
    static const bool attr_ = (cudaFuncSetAttribute(k_solve_bwd<T, NR>,                     \
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                                    kSolveSmemBytes),                             \
                               true);                                                             \
    (void)attr_;                                                                                  \
    k_solve_bwd<T, NR><<<nf, threads, sm, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff, use);\
  } while (0)
  if (nrhs == 1) MFGPU_BWD(1);
  else if (nrhs <= 4) MFGPU_BWD(4);
  else if (nrhs <= 8) MFGPU_BWD(8);
  else MFGPU_BWD(16);
#undef MFGPU_BWD
  g_launches++;
}

template <class T>
void launch_root_solve(int f, int N, const FrontDev* fr, const T* F, const int* dofs, T* X,
                       int64_t ldx, int nrhs, T* W, const int64_t* woff, cudaStream_t st) {
  size_t sm;
  int use;
  smemFor(N, nrhs, sizeof(T), sm, use);
#define MFGPU_ROOT(NR)                                                                          \
  do {                                                                                          \
    static const bool attr_ = (cudaFuncSetAttribute(k_root_solve<T, NR>,                     \
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                                    kSolveSmemBytes),                             \
                               true);                                                             \
    (void)attr_;                                                                                  \
    k_root_solve<T, NR><<<1, ST, sm, st>>>(f, fr, F, dofs, X, ldx, nrhs, W, woff, use);         \
  } while (0)
  if (nrhs == 1) MFGPU_ROOT(1);
  else if (nrhs <= 4) MFGPU_ROOT(4);
  else if (nrhs <= 8) MFGPU_ROOT(8);
  else MFGPU_ROOT(16);
#undef MFGPU_ROOT
  g_launches++;
}

template <class T>
void launch_apply_up(const int* flist, int nf, const FrontDev* fr, const T* F, const int* dofs, T* X,
                     int64_t ldx, int nrhs, T* W, const int64_t* woff, T* Tb, cudaStream_t st) {
  if (nf <= 0) return;
  k_apply_up<T><<<nf, ST, 0, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff, Tb);
  g_launches++;
}
template <class T>
void launch_apply_down(const int* flist, int nf, const FrontDev* fr, const T* F, const int* dofs,
                       int64_t ldx, int nrhs, T* W, const int64_t* woff, const T* Tb,
                       cudaStream_t st) {
  if (nf <= 0) return;
  k_apply_down<T><<<nf, ST, 0, st>>>(flist, fr, F, dofs, ldx, nrhs, W, woff, Tb);
  g_launches++;
}
template <class T>
void launch_root_apply(int f, const FrontDev* fr, const T* F, const int* dofs, T* X, int64_t ldx,
                       int nrhs, T* W, const int64_t* woff, cudaStream_t st) {
  k_root_apply<T><<<1, ST, 0, st>>>(f, fr, F, dofs, X, ldx, nrhs, W, woff);
  g_launches++;
}
template <class T>
void launch_sep_gather(const int* slist, int ns, const SepDev* sp, const int* dofs, T* X,
                       int64_t ldx, int nrhs, const T* W, const int64_t* woff, const FrontDev* fr,
                       cudaStream_t st) {
  if (ns <= 0) return;
  k_sep_gather<T><<<ns, ST, 0, st>>>(slist, sp, dofs, X, ldx, nrhs, W, woff, fr);
  g_launches++;
}

void launch_lu_solve(bool forward, const int* flist, int nf, int maxN, const FrontDev* fr,
                     const double* F, const int* ipiv, const int* dofs, double* X, int64_t ldx,
                     int nrhs, double* W, const int64_t* woff, cudaStream_t st) {
  if (nf <= 0) return;
  size_t sm;
  int use;
  smemFor(maxN, nrhs, sizeof(double), sm, use);
  const int threads = sweep_threads(maxN);
#define MFGPU_LU(NR)                                                                             \
  do {                                                                                           \
    if (forward) {                                                                               \
      static const bool attr_ = (cudaFuncSetAttribute(k_lu_solve_fwd<NR>,                        \
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                                      kSolveSmemBytes),                            \
                                 true);                                                            \
      (void)attr_;                                                                               \
      k_lu_solve_fwd<NR><<<nf, threads, sm, st>>>(flist, fr, F, ipiv, dofs, X, ldx, nrhs, W, woff, \
                                                  use);                                          \
    } else {                                                                                     \
      static const bool attr_ = (cudaFuncSetAttribute(k_lu_solve_bwd<NR>,                        \
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                                      kSolveSmemBytes),                            \
                                 true);                                                            \
      (void)attr_;                                                                               \
      k_lu_solve_bwd<NR><<<nf, threads, sm, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff, use); \
    }                                                                                            \
  } while (0)
  if (nrhs == 1) MFGPU_LU(1);
  else if (nrhs <= 4) MFGPU_LU(4);
  else if (nrhs <= 8) MFGPU_LU(8);
  else MFGPU_LU(16);
#undef MFGPU_LU
  g_launches++;
}

void launch_lu_apply_up(const int* flist, int nf, const FrontDev* fr, const double* F,
                        const int* ipiv, const int* dofs, double* X, int64_t ldx, int nrhs,
                        double* W, const int64_t* woff, double* Tb, cudaStream_t st) {
  if (nf <= 0) return;
  k_lu_apply_up<<<nf, ST, 0, st>>>(flist, fr, F, ipiv, dofs, X, ldx, nrhs, W, woff, Tb);
  g_launches++;
}

template <class T>
cudaError_t launch_trail_syrk(const int* flist, int nf, const FrontDev* fr, T* F, int Ks, int w,
                              cudaStream_t st) {
  if (nf <= 0) return cudaSuccess;
  if (nf > kMaxPanelFronts || w <= 0) return cudaErrorInvalidValue;
  const size_t sm = 2 * 64 * kPS * sizeof(T);
  static const int grid = [sm]() {   // thread-safe one-time set-up: every resident CTA
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_trail_syrk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trail_syrk<T>, kCT, sm);
    return sms * std::max(1, per);
  }();
  k_trail_syrk<T><<<grid, kCT, sm, st>>>(flist, nf, fr, F, Ks, w);
  g_launches++;
  return cudaGetLastError();
}

#define MFGPU_INSTANTIATE(T)                                                                      \
  template void launch_tasks<T>(const Task*, const int64_t*, int, int64_t, T*, T*, const int*,     \
                                const int*, const double*, const int*, const double*, cudaStream_t); \
  template cudaError_t launch_level_coop<T>(const int*, int, int, const FrontDev*, T*, DevError*,  \
                                            T*, const int*, unsigned*, cudaStream_t, int, int, int, \
                                            int, int, int);                                         \
  template void launch_front_small<T>(const int*, int, int, const FrontDev*, T*, DevError*,        \
                                      cudaStream_t);                                                \
  template void launch_solve_fwd<T>(const int*, int, int, const FrontDev*, const T*, const int*,   \
                                    T*, int64_t, int, T*, const int64_t*, cudaStream_t);            \
  template void launch_solve_bwd<T>(const int*, int, int, const FrontDev*, const T*, const int*,   \
                                    T*, int64_t, int, T*, const int64_t*, cudaStream_t);            \
  template void launch_root_solve<T>(int, int, const FrontDev*, const T*, const int*, T*, int64_t, \
                                     int, T*, const int64_t*, cudaStream_t);                        \
  template void launch_apply_up<T>(const int*, int, const FrontDev*, const T*, const int*, T*,     \
                                   int64_t, int, T*, const int64_t*, T*, cudaStream_t);             \
  template void launch_apply_down<T>(const int*, int, const FrontDev*, const T*, const int*,       \
                                     int64_t, int, T*, const int64_t*, const T*, cudaStream_t);     \
  template void launch_root_apply<T>(int, const FrontDev*, const T*, const int*, T*, int64_t, int, \
                                     T*, const int64_t*, cudaStream_t);                             \
  template void launch_sep_gather<T>(const int*, int, const SepDev*, const int*, T*, int64_t, int, \
                                     const T*, const int64_t*, const FrontDev*, cudaStream_t);      \
  template cudaError_t launch_trail_syrk<T>(const int*, int, const FrontDev*, T*, int, int,       \
                                            cudaStream_t);

MFGPU_INSTANTIATE(double)
MFGPU_INSTANTIATE(float)
#undef MFGPU_INSTANTIATE

}  // namespace mfgpu
