// FP64 kernels: front / separator assembly from task tables, panel-stepped
// partial Cholesky of every front of a level, and the solve / apply sweeps.
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

#include <atomic>
#include <cstdio>

#include "device.cuh"

namespace cg = cooperative_groups;

namespace mfgpu {

std::atomic<long long> g_launches{0};

namespace {

__device__ __forceinline__ double sparse_at(const int* __restrict__ rp, const int* __restrict__ ci,
                                            const double* __restrict__ va, int r, int c) {
  // Sparse<Scalar>::operator()(i, j) (src/LinAlg/sparse.cpp:80-92): scan row r.
  int p = rp[r], e = rp[r + 1];
  double v = 0.0;
  for (; p < e; p++)
    if (ci[p] == c) v = va[p];
  return v;
}

__global__ void __launch_bounds__(256) k_tasks(const Task* __restrict__ tasks,
                                               const int64_t* __restrict__ tstart, int ntasks,
                                               double* __restrict__ F, double* __restrict__ SA,
                                               const int* __restrict__ rp,
                                               const int* __restrict__ ci,
                                               const double* __restrict__ va,
                                               const int* __restrict__ dofs) {
  __shared__ double sm[kTaskTile][kTaskTile + 1];
  __shared__ int s_task;
  const int64_t tile = (int64_t)blockIdx.x + (int64_t)blockIdx.y * gridDim.x;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    int lo = 0, hi = ntasks - 1;   // last t with tstart[t] <= tile
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (tstart[mid] <= tile) lo = mid;
      else hi = mid - 1;
    }
    s_task = lo;
  }
  __syncthreads();
  if (tile >= tstart[ntasks]) return;
  const Task T = tasks[s_task];
  const int64_t local = tile - tstart[s_task];
  const int tr = (T.rows + kTaskTile - 1) / kTaskTile;
  const int i0 = (int)(local % tr) * kTaskTile;
  const int j0 = (int)(local / tr) * kTaskTile;
  if (T.lower && i0 + kTaskTile - 1 < j0) return;
  double* dst = (T.dst_arena == AR_FRONT ? F : SA) + T.dst_off;
  const double* src = (T.src_arena == AR_FRONT ? F : SA) + T.src_off;
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (T.kind == TK_COPY && T.trans) {
    // dst(i, j) = src[j + i*ld]: stage through shared memory so both sides coalesce
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int ii = i0 + ty + 8 * q, jj = j0 + tx;
      if (ii < T.rows && jj < T.cols) sm[ty + 8 * q][tx] = src[jj + (int64_t)ii * T.src_ld];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int i = i0 + tx, j = j0 + ty + 8 * q;
      if (i < T.rows && j < T.cols && (!T.lower || i >= j))
        dst[i + (int64_t)j * T.dst_ld] = sm[tx][ty + 8 * q];
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = i0 + tx, j = j0 + ty + 8 * q;
    if (i >= T.rows || j >= T.cols || (T.lower && i < j)) continue;
    double* d = dst + i + (int64_t)j * T.dst_ld;
    switch (T.kind) {
      case TK_ZERO: *d = 0.0; break;
      case TK_COPY: *d = src[i + (int64_t)j * T.src_ld]; break;
      case TK_ADD: *d = *d + src[i + (int64_t)j * T.src_ld]; break;
      case TK_SPARSE: *d = sparse_at(rp, ci, va, dofs[T.row_dof + i], dofs[T.col_dof + j]); break;
    }
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
__device__ void warp_factor_inv(double* A, int64_t ld, int k, int kb, double (*Ls)[kPanel + 1],
                                double* Li, double* Dinv, DevError* err, int f) {
  const int lane = threadIdx.x & 31;
  double row[kPanel];
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    row[t] = (lane < kb && t < kb && t <= lane) ? A[(k + lane) + (int64_t)(k + t) * ld] : 0.0;
  int bad = -1;
#pragma unroll
  for (int j = 0; j < kPanel; j++) {
    if (j < kb) {
      double s0 = row[j], s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
      for (int t = 0; t < j; t++) {
        const double l = Ls[j][t];
        if ((t & 3) == 0) s0 -= row[t] * l;
        else if ((t & 3) == 1) s1 -= row[t] * l;
        else if ((t & 3) == 2) s2 -= row[t] * l;
        else s3 -= row[t] * l;
      }
      const double sv = (s0 + s1) + (s2 + s3);
      double piv = __shfl_sync(kFull, sv, j);
      if (!(piv > 0.0)) {                // non-positive or NaN pivot: not SPD
        if (bad < 0) bad = j;
        piv = 1.0;
      }
      const double r = rsqrt(piv);
      row[j] = lane == j ? piv * r : (lane > j ? sv * r : 0.0);
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
  double x[kPanel];
#pragma unroll
  for (int i = 0; i < kPanel; i++) {
    double v = 0.0;
    if (i < kb) {
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
      for (int t = 0; t < i; t++) {
        const double l = Ls[i][t];
        const double xt = t >= lane ? x[t] : 0.0;
        if ((t & 3) == 0) s0 += l * xt;
        else if ((t & 3) == 1) s1 += l * xt;
        else if ((t & 3) == 2) s2 += l * xt;
        else s3 += l * xt;
      }
      const double di = Dinv[i];
      v = i == lane ? di : (i > lane ? -((s0 + s1) + (s2 + s3)) * di : 0.0);
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
constexpr int kSmallMaxN = 640;  // widest front the fused kernel handles (panel in smem)

// acc(32x32) = X[I0:I0+32, 0:kk] * Y[J0:J0+32, 0:kk]^T for row-major operands
// in shared memory (strides sx, sy; rows padded with zeros to the tile edge).
__device__ __forceinline__ void warp_gemm_nt(const double* X, int sx, int I0, const double* Y, int sy,
                                             int J0, int kk, int lane, double (&acc)[4][4][2]) {
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
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

__device__ __forceinline__ void warp_syrk_tile(const double* P, int I0, int J0, int kk, int lane,
                                               double (&acc)[4][4][2]) {
  warp_gemm_nt(P, kPS, I0, P, kPS, J0, kk, lane, acc);
}

// Panel triangular solve of the 32-row block R0 of P in place with the explicit
// inverse: P(R0 block) <- P(R0 block) Li^T; rows < M are also written to A at
// (r0 + row, k + col), cols < kb.
__device__ __forceinline__ void warp_trsm_block(double* P, int R0, const double* Li, int kb,
                                                double* A, int64_t ld, int r0, int k, int M,
                                                int lane) {
  double acc[4][4][2];
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
__device__ __forceinline__ void warp_tile_sub(double* A, int64_t ld, int r0, int M, int I0, int J0,
                                              int lane, const double (&acc)[4][4][2]) {
  const int rr = lane >> 2, cc = lane & 3;
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int j = J0 + 8 * b + 2 * cc + q;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int i = I0 + 8 * a + rr;
        if (i < M && j < M && i >= j) A[(r0 + i) + (int64_t)(r0 + j) * ld] -= acc[a][b][q];
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
__global__ void __launch_bounds__(256) k_front_small(const int* __restrict__ flist,
                                                     const FrontDev* __restrict__ fr,
                                                     double* __restrict__ F, DevError* err) {
  extern __shared__ double Psm[];
  __shared__ double Ls[kPanel][kPanel + 1];
  __shared__ double Li[kPanel * kLi];
  __shared__ double Dinv[kPanel];
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* A = F + d.off;
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
      Psm[rr * kPS + t] = (rr < M && t < kb) ? A[(r0 + rr) + (int64_t)(k + t) * ld] : 0.0;
    }
    __syncthreads();
    for (int R0 = warp * 32; R0 < Mp; R0 += 256) warp_trsm_block(Psm, R0, Li, kb, A, ld, r0, k, M, lane);
    __syncthreads();
    const int T = Mp >> 5;
    const int ntile = T * (T + 1) / 2;
    const int kk = (kb + 3) & ~3;
    if (warp == 0) {
      // lookahead: tile (0, 0) holds the next diagonal block; update it, then
      // factor it while the other warps finish the trailing update
      if (ntile > 0) {
        double acc[4][4][2];
        warp_syrk_tile(Psm, 0, 0, kk, lane, acc);
        warp_tile_sub(A, ld, r0, M, 0, 0, lane, acc);
      }
      __syncwarp();
      if (r0 < d.n) warp_factor_inv(A, ld, r0, min(kPanel, d.n - r0), Ls, Li, Dinv, err, f);
    } else {
      for (int t = warp; t < ntile; t += 7) {   // warps 1..7 take tiles 1, 2, ...
        int I, J;
        tri_index(t, I, J);
        double acc[4][4][2];
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
// blocking: outer panels of kOuter columns; inside each, 32-column steps
//   A  triangular solve of the rows below the diagonal block (every work item
//      factors the 32 x 32 diagonal block itself, from the not yet overwritten
//      values, so no extra phase is needed),
//   B  the diagonal block is written back and the outer panel's remaining
//      columns are updated with the 32 new columns,
// and after the outer panel
//   C  the trailing matrix is updated with the whole outer panel (k = kOuter).
// Phases are separated by grid-wide barriers; work items (row blocks, 64 x 64
// tiles) of all fronts of the level are spread over all CTAs.
// ---------------------------------------------------------------------------
constexpr int kOuter = 256;
constexpr int kCT = 128;           // threads per CTA of the cooperative kernel
constexpr int kMaxCoopFronts = 256;

// C(tile) -= X(rows) X(cols)^T over columns [k0, k1) of the front, 64 x 64 tile
// at rows [ri, ri+64), cols [ci, ci+64); rows < N, cols < cmax, row >= col.
__device__ void coop_tile_update(double* A, int64_t ld, int N, int cmax, int ri, int ci, int k0,
                                 int k1, double* Xa, double* Xb) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wi = warp >> 1, wj = warp & 1;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
  const bool diag = (ri == ci);
  const bool live = !(diag && wi < wj);
  for (int kc = k0; kc < k1; kc += kPanel) {
    const int kb = min(kPanel, k1 - kc);
    __syncthreads();
    for (int idx = tid; idx < 64 * kPanel; idx += kCT) {
      const int i = idx % 64, t = idx / 64;
      const bool ok = t < kb;
      const int ra = ri + i, rb = ci + i;
      Xa[i * kPS + t] = (ok && ra < N) ? A[ra + (int64_t)(kc + t) * ld] : 0.0;
      Xb[i * kPS + t] = (ok && rb < N) ? A[rb + (int64_t)(kc + t) * ld] : 0.0;
    }
    __syncthreads();
    if (live) {
      const int rr = lane >> 2, cc = lane & 3;
      const int kk = (kb + 3) & ~3;
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
  }
  if (!live) return;
  const int rr = lane >> 2, cc = lane & 3;
#pragma unroll
  for (int b = 0; b < 4; b++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int c = ci + wj * 32 + 8 * b + 2 * cc + q;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int r = ri + wi * 32 + 8 * a + rr;
        if (r < N && c < cmax && r >= c) A[r + (int64_t)c * ld] -= acc[a][b][q];
      }
    }
}

// Factored diagonal blocks are handed from the CTA that completes their update
// to every work item of the next step through a per-front slot in global
// memory holding the inverse of the factor (32 rows of stride kLi).
constexpr int kDiagSlot = kPanel * kLi;

// Warp 0 of the calling CTA factors the diagonal block at (k, k), writes it
// back into the front and publishes it in `slot`.  Every thread must call.
__device__ void coop_factor_publish(double* A, int64_t ld, int k, int kb, double* slot,
                                    double (*Ls)[kPanel + 1], double* Li, double* Dinv,
                                    DevError* err, int f) {
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    warp_factor_inv(A, ld, k, kb, Ls, Li, Dinv, err, f);
    for (int i = 0; i < kPanel; i++) slot[i * kLi + lane] = Li[i * kLi + lane];
  }
}

__device__ __forceinline__ int ceil_div(int a, int b) { return (a + b - 1) / b; }

__global__ void __launch_bounds__(kCT) k_level_coop(const int* __restrict__ flist, int nf,
                                                    const FrontDev* __restrict__ fr,
                                                    double* __restrict__ F, DevError* err, int maxn,
                                                    double* __restrict__ slots) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double Ls[kPanel][kPanel + 1];
  __shared__ double Li[kPanel * kLi];
  __shared__ double Dinv[kPanel];
  extern __shared__ double Xab[];   // 2 * 64 * kPS doubles (dynamic)
  __shared__ int pre[kMaxCoopFronts + 1];
  double* Xa = Xab;             // phase B / C tile operands
  double* Xb = Xab + 64 * kPS;
  double* Rows = Xab;           // phase A: kCT = 128 staged rows
  const int tid = threadIdx.x;
  // the first diagonal block of every front
  for (int i = blockIdx.x; i < nf; i += gridDim.x) {
    const int f = flist[i];
    const FrontDev d = fr[f];
    if (d.n > 0)
      coop_factor_publish(F + d.off, d.ld, 0, min(kPanel, d.n), slots + (int64_t)i * kDiagSlot, Ls,
                          Li, Dinv, err, f);
  }
  grid.sync();
  for (int K = 0; K < maxn; K += kOuter) {
    for (int k = K; k < K + kOuter && k < maxn; k += kPanel) {
      // ---- phase A: rows below the (already factored) diagonal block ----
      __syncthreads();
      if (tid == 0) {
        pre[0] = 0;
        for (int i = 0; i < nf; i++) {
          const FrontDev d = fr[flist[i]];
          int c = 0;
          if (k < d.n) c = ceil_div(d.N - k - min(kPanel, d.n - k), kCT);
          pre[i + 1] = pre[i] + c;
        }
      }
      __syncthreads();
      for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
        int i = 0;
        while (pre[i + 1] <= item) i++;
        const FrontDev d = fr[flist[i]];
        double* A = F + d.off;
        const int kb = min(kPanel, d.n - k);
        const double* slot = slots + (int64_t)i * kDiagSlot;
        const int rbase = k + kb + (item - pre[i]) * kCT;
        const int Mi = min(kCT, d.N - rbase);
        __syncthreads();
        for (int idx = tid; idx < kPanel * kLi; idx += kCT) Li[idx] = slot[idx];
        for (int idx = tid; idx < kCT * kPanel; idx += kCT) {
          const int rr = idx % kCT, t = idx / kCT;
          Rows[rr * kPS + t] = (rr < Mi && t < kb) ? A[(rbase + rr) + (int64_t)(k + t) * d.ld] : 0.0;
        }
        __syncthreads();
        warp_trsm_block(Rows, (tid >> 5) * 32, Li, kb, A, d.ld, rbase, k, Mi, tid & 31);
      }
      grid.sync();
      // ---- phase B: update the outer panel's remaining columns; the CTA that
      // updates the next diagonal block factors and publishes it ----
      __syncthreads();
      if (tid == 0) {
        pre[0] = 0;
        for (int i = 0; i < nf; i++) {
          const FrontDev d = fr[flist[i]];
          int c = 0;
          if (k < d.n) {
            const int kb = min(kPanel, d.n - k);
            const int c0 = k + kb, cmax = min(K + kOuter, d.n);
            if (cmax > c0) {
              const int TI = ceil_div(d.N - c0, 64), TJ = ceil_div(cmax - c0, 64);
              for (int J = 0; J < TJ; J++) c += TI - J;
            }
          }
          pre[i + 1] = pre[i] + c;
        }
      }
      __syncthreads();
      for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
        int i = 0;
        while (pre[i + 1] <= item) i++;
        const int f = flist[i];
        const FrontDev d = fr[f];
        double* A = F + d.off;
        const int kb = min(kPanel, d.n - k);
        int local = item - pre[i];
        const int c0 = k + kb, cmax = min(K + kOuter, d.n);
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
      grid.sync();
    }
    // ---- phase C: trailing update with the outer panel ----
    __syncthreads();
    if (tid == 0) {
      pre[0] = 0;
      for (int i = 0; i < nf; i++) {
        const FrontDev d = fr[flist[i]];
        int c = 0;
        const int k1 = min(K + kOuter, d.n);
        if (K < d.n && d.N > k1) {
          const int T = ceil_div(d.N - k1, 64);
          c = T * (T + 1) / 2;
        }
        pre[i + 1] = pre[i] + c;
      }
    }
    __syncthreads();
    for (int item = blockIdx.x; item < pre[nf]; item += gridDim.x) {
      int i = 0;
      while (pre[i + 1] <= item) i++;
      const int f = flist[i];
      const FrontDev d = fr[f];
      const int k1 = min(K + kOuter, d.n);
      int I, J;
      tri_index(item - pre[i], I, J);
      coop_tile_update(F + d.off, d.ld, d.N, d.N, k1 + I * 64, k1 + J * 64, K, k1, Xa, Xb);
      if (I == 0 && J == 0 && k1 < d.n)
        coop_factor_publish(F + d.off, d.ld, k1, min(kPanel, d.n - k1), slots + (int64_t)i * kDiagSlot,
                            Ls, Li, Dinv, err, f);
    }
    grid.sync();
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
template <int NR>
__device__ void front_forward(const FrontDev& d, const double* __restrict__ A, double* W,
                              int nrhs) {
  __shared__ double Ls[kPanel][kPanel + 1];
  __shared__ double xs[kPanel][NR + 1];
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
        if (lane == j) {
          const double djj = Ls[j][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[j][c] = xs[j][c] / djj;
        }
        __syncwarp();
        if (lane > j && lane < kb) {
          const double l = Ls[lane][j];
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
      double acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = 0.0;
      const double* Lr = A + r + (int64_t)k * ld;
      if (kb == kPanel) {
        // all 32 loads issued before the FMAs: memory-level parallelism
        double l[kPanel];
#pragma unroll
        for (int t = 0; t < kPanel; t++) l[t] = Lr[(int64_t)t * ld];
#pragma unroll
        for (int t = 0; t < kPanel; t++)
#pragma unroll
          for (int c = 0; c < NR; c++) acc[c] = fma(l[t], xs[t][c], acc[c]);
      } else {
        for (int t = 0; t < kb; t++) {
          const double l = Lr[(int64_t)t * ld];
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
template <int NR>
__device__ void front_backward(const FrontDev& d, const double* __restrict__ A, double* W,
                               int nrhs) {
  __shared__ double Ls[kPanel][kPanel + 1];
  __shared__ double xs[kPanel][NR + 1];
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
      double acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = 0.0;
      const double* Lc = A + (int64_t)(k + j) * ld;
      int r = k + kb + lane;
      for (; r + 96 < N; r += 128) {      // four independent loads in flight
        const double l0 = Lc[r], l1 = Lc[r + 32], l2 = Lc[r + 64], l3 = Lc[r + 96];
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) {
            const double* w = W + (int64_t)c * N + r;
            acc[c] = fma(l0, w[0], acc[c]);
            acc[c] = fma(l1, w[32], acc[c]);
            acc[c] = fma(l2, w[64], acc[c]);
            acc[c] = fma(l3, w[96], acc[c]);
          }
      }
      for (; r < N; r += 32) {
        const double l = Lc[r];
#pragma unroll
        for (int c = 0; c < NR; c++)
          if (c < nrhs) acc[c] = fma(l, W[r + (int64_t)c * N], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < NR; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && c < nrhs) xs[j][c] = W[k + j + (int64_t)c * N] - v;
      }
    }
    __syncthreads();
    if (warp == 0) {
      for (int j = kb - 1; j >= 0; j--) {
        if (lane == j) {
          const double djj = Ls[j][j];
#pragma unroll
          for (int c = 0; c < NR; c++)
            if (c < nrhs) xs[j][c] = xs[j][c] / djj;
        }
        __syncwarp();
        if (lane < j) {
          const double l = Ls[j][lane];
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

template <int NR>
__global__ void __launch_bounds__(ST) k_solve_fwd(const int* __restrict__ flist,
                                                  const FrontDev* __restrict__ fr,
                                                  const double* __restrict__ F,
                                                  const int* __restrict__ dofs, double* X,
                                                  int64_t ldx, int nrhs, double* Wb,
                                                  const int64_t* __restrict__ woff, int use_smem) {
  extern __shared__ double smW[];
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* Wg = Wb + woff[f] * nrhs;
  double* W = use_smem ? smW : Wg;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = i < d.n ? X[dl[i] + (int64_t)c * ldx] : 0.0;
  }
  __syncthreads();
  front_forward<NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    if (i < d.n) X[dl[i] + (int64_t)c * ldx] = W[idx];
    else if (use_smem) Wg[idx] = W[idx];    // boundary part for the separator gather
  }
}

template <int NR>
__global__ void __launch_bounds__(ST) k_solve_bwd(const int* __restrict__ flist,
                                                  const FrontDev* __restrict__ fr,
                                                  const double* __restrict__ F,
                                                  const int* __restrict__ dofs, double* X,
                                                  int64_t ldx, int nrhs, double* Wb,
                                                  const int64_t* __restrict__ woff, int use_smem) {
  extern __shared__ double smW[];
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = use_smem ? smW : Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  front_backward<NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

template <int NR>
__global__ void __launch_bounds__(ST) k_root_solve(int f, const FrontDev* __restrict__ fr,
                                                   const double* __restrict__ F,
                                                   const int* __restrict__ dofs, double* X,
                                                   int64_t ldx, int nrhs, double* Wb,
                                                   const int64_t* __restrict__ woff, int use_smem) {
  extern __shared__ double smW[];
  const FrontDev d = fr[f];
  double* W = use_smem ? smW : Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  front_forward<NR>(d, F + d.off, W, nrhs);
  front_backward<NR>(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

// X(sep) = (X(sep) + W_box0(sep rows)) + W_box1(sep rows), the reference's
// per-box accumulation order (mf2d.cpp:992-1011, 1036-1047).
__global__ void __launch_bounds__(ST) k_sep_gather(const int* __restrict__ slist,
                                                   const SepDev* __restrict__ sp,
                                                   const int* __restrict__ dofs, double* X,
                                                   int64_t ldx, int nrhs,
                                                   const double* __restrict__ Wb,
                                                   const int64_t* __restrict__ woff,
                                                   const FrontDev* __restrict__ fr) {
  const SepDev s = sp[slist[blockIdx.x]];
  const int* dl = dofs + s.dof_off;
  const int N0 = fr[s.box0].N, N1 = fr[s.box1].N;
  const double* W0 = Wb + woff[s.box0] * nrhs;
  const double* W1 = Wb + woff[s.box1] * nrhs;
  for (int idx = threadIdx.x; idx < s.s * nrhs; idx += blockDim.x) {
    const int i = idx % s.s, c = idx / s.s;
    double* x = X + dl[i] + (int64_t)c * ldx;
    *x = (*x + W0[s.pos0 + i + (int64_t)c * N0]) + W1[s.pos1 + i + (int64_t)c * N1];
  }
}

// Apply, upward part: t = L11^T b_piv + L21^T b_bd ; b_piv = L11 t ; T(piv) = t.
__device__ void front_apply_up(const FrontDev& d, const double* __restrict__ A, double* W,
                               double* Tt, int nrhs) {
  // W holds [b_piv; b_bd] (N x nrhs); Tt receives t (n x nrhs, ld n).
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int jc = warp; jc < n * nrhs; jc += nw) {
    const int j = jc % n, c = jc / n;
    const double* w = W + (int64_t)c * N;
    double s = 0.0;
    for (int r = j + lane; r < N; r += 32) s += A[r + (int64_t)j * ld] * w[r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) Tt[j + (int64_t)c * n] = s;
  }
  __syncthreads();
  for (int idx = tid; idx < n * nrhs; idx += blockDim.x) {
    const int r = idx % n, c = idx / n;
    const double* t = Tt + (int64_t)c * n;
    double s = 0.0;
    for (int j = 0; j <= r; j++) s += A[r + (int64_t)j * ld] * t[j];
    W[r + (int64_t)c * N] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(ST) k_apply_up(const int* __restrict__ flist,
                                                 const FrontDev* __restrict__ fr,
                                                 const double* __restrict__ F,
                                                 const int* __restrict__ dofs, double* X,
                                                 int64_t ldx, int nrhs, double* Wb,
                                                 const int64_t* __restrict__ woff, double* T) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  double* Tt = W + (int64_t)d.N * nrhs;  // second half of the front's workspace
  front_apply_up(d, F + d.off, W, Tt, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
    T[dl[i] + (int64_t)c * ldx] = Tt[i + (int64_t)c * d.n];
  }
}

// Apply, downward part: W[n,N) = L21 t (t read from T by DOF).
__global__ void __launch_bounds__(ST) k_apply_down(const int* __restrict__ flist,
                                                   const FrontDev* __restrict__ fr,
                                                   const double* __restrict__ F,
                                                   const int* __restrict__ dofs, int64_t ldx,
                                                   int nrhs, double* Wb,
                                                   const int64_t* __restrict__ woff,
                                                   const double* __restrict__ T) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  const double* A = F + d.off;
  double* Tt = W + (int64_t)d.N * nrhs;
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    Tt[i + (int64_t)c * d.n] = T[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < d.m * nrhs; idx += blockDim.x) {
    const int r = d.n + idx % d.m, c = idx / d.m;
    const double* t = Tt + (int64_t)c * d.n;
    double s = 0.0;
    for (int j = 0; j < d.n; j++) s += A[r + (int64_t)j * d.ld] * t[j];
    W[r + (int64_t)c * d.N] = s;
  }
}

__global__ void __launch_bounds__(ST) k_root_apply(int f, const FrontDev* __restrict__ fr,
                                                   const double* __restrict__ F,
                                                   const int* __restrict__ dofs, double* X,
                                                   int64_t ldx, int nrhs, double* Wb,
                                                   const int64_t* __restrict__ woff) {
  const FrontDev d = fr[f];
  double* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  double* Tt = W + (int64_t)d.N * nrhs;
  front_apply_up(d, F + d.off, W, Tt, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

}  // namespace

void launch_tasks(const Task* tasks, const int64_t* tstart, int ntasks, int64_t ntiles,
                  double* fronts, double* seps, const int* rp, const int* ci, const double* va,
                  const int* dofs, cudaStream_t st) {
  if (ntasks <= 0 || ntiles <= 0) return;
  const int64_t gx = ntiles < 65535 * 32 ? ntiles : 65535 * 32;
  const int64_t gy = (ntiles + gx - 1) / gx;
  k_tasks<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(tasks, tstart, ntasks, fronts,
                                                                      seps, rp, ci, va, dofs);
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

bool small_front_fits(int maxN) { return maxN <= kSmallMaxN; }

bool coop_fits(int nf) { return nf <= kMaxCoopFronts; }
size_t coop_slot_doubles() { return (size_t)kMaxCoopFronts * kDiagSlot; }

cudaError_t launch_level_coop(const int* flist, int nf, int maxn, const FrontDev* fr, double* F,
                              DevError* err, double* slots, cudaStream_t st) {
  if (nf <= 0) return cudaSuccess;
  const size_t sm = 2 * 64 * kPS * sizeof(double);
  static int grid = 0;   // co-resident CTAs on this device (same for every call)
  if (grid == 0) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_level_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_level_coop, kCT, sm);
    grid = sms * (per > 0 ? per : 1);
  }
  void* args[] = {(void*)&flist, (void*)&nf, (void*)&fr, (void*)&F, (void*)&err, (void*)&maxn,
                  (void*)&slots};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_level_coop, dim3(grid), dim3(kCT), args,
                                              sm, st);
  g_launches++;
  return e;
}

void launch_front_small(const int* flist, int nf, int maxN, const FrontDev* fr, double* F,
                        DevError* err, cudaStream_t st) {
  if (nf <= 0) return;
  const size_t sm = (size_t)((maxN + 31) & ~31) * kPS * sizeof(double);
  cudaFuncSetAttribute(k_front_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_front_small<<<nf, 256, sm, st>>>(flist, fr, F, err);
  g_launches++;
}

// Solve kernels are templated on a bound of the right-hand-side count and keep
// the front's right-hand-side block in dynamic shared memory when the largest
// front's fits.
namespace {
template <int NR>
void fwd_launch(int grid, size_t sm, int use, cudaStream_t st, const int* fl, const FrontDev* fr,
                const double* F, const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                const int64_t* woff) {
  if (sm) cudaFuncSetAttribute(k_solve_fwd<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_solve_fwd<NR><<<grid, ST, sm, st>>>(fl, fr, F, dofs, X, ldx, nrhs, W, woff, use);
}
template <int NR>
void bwd_launch(int grid, size_t sm, int use, cudaStream_t st, const int* fl, const FrontDev* fr,
                const double* F, const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                const int64_t* woff) {
  if (sm) cudaFuncSetAttribute(k_solve_bwd<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_solve_bwd<NR><<<grid, ST, sm, st>>>(fl, fr, F, dofs, X, ldx, nrhs, W, woff, use);
}
template <int NR>
void root_launch(size_t sm, int use, cudaStream_t st, int f, const FrontDev* fr, const double* F,
                 const int* dofs, double* X, int64_t ldx, int nrhs, double* W, const int64_t* woff) {
  if (sm) cudaFuncSetAttribute(k_root_solve<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_root_solve<NR><<<1, ST, sm, st>>>(f, fr, F, dofs, X, ldx, nrhs, W, woff, use);
}
void smemFor(int maxN, int nrhs, size_t& sm, int& use) {
  const size_t need = (size_t)maxN * nrhs * sizeof(double);
  use = need <= (size_t)kSolveSmemBytes;
  sm = use ? need : 0;
}
}  // namespace

void launch_solve_fwd(const int* flist, int nf, int maxN, const FrontDev* fr, const double* F,
                      const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                      const int64_t* woff, cudaStream_t st) {
  if (nf <= 0) return;
  size_t sm;
  int use;
  smemFor(maxN, nrhs, sm, use);
  if (nrhs == 1) fwd_launch<1>(nf, sm, use, st, flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  else if (nrhs <= 4) fwd_launch<4>(nf, sm, use, st, flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  else fwd_launch<16>(nf, sm, use, st, flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  g_launches++;
}
void launch_solve_bwd(const int* flist, int nf, int maxN, const FrontDev* fr, const double* F,
                      const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                      const int64_t* woff, cudaStream_t st) {
  if (nf <= 0) return;
  size_t sm;
  int use;
  smemFor(maxN, nrhs, sm, use);
  if (nrhs == 1) bwd_launch<1>(nf, sm, use, st, flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  else if (nrhs <= 4) bwd_launch<4>(nf, sm, use, st, flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  else bwd_launch<16>(nf, sm, use, st, flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  g_launches++;
}
void launch_apply_up(const int* flist, int nf, const FrontDev* fr, const double* F,
                     const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                     const int64_t* woff, double* T, cudaStream_t st) {
  if (nf <= 0) return;
  k_apply_up<<<nf, ST, 0, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff, T);
  g_launches++;
}
void launch_apply_down(const int* flist, int nf, const FrontDev* fr, const double* F,
                       const int* dofs, int64_t ldx, int nrhs, double* W, const int64_t* woff,
                       const double* T, cudaStream_t st) {
  if (nf <= 0) return;
  k_apply_down<<<nf, ST, 0, st>>>(flist, fr, F, dofs, ldx, nrhs, W, woff, T);
  g_launches++;
}
void launch_root_solve(int f, int N, const FrontDev* fr, const double* F, const int* dofs,
                       double* X, int64_t ldx, int nrhs, double* W, const int64_t* woff,
                       cudaStream_t st) {
  size_t sm;
  int use;
  smemFor(N, nrhs, sm, use);
  if (nrhs == 1) root_launch<1>(sm, use, st, f, fr, F, dofs, X, ldx, nrhs, W, woff);
  else if (nrhs <= 4) root_launch<4>(sm, use, st, f, fr, F, dofs, X, ldx, nrhs, W, woff);
  else root_launch<16>(sm, use, st, f, fr, F, dofs, X, ldx, nrhs, W, woff);
  g_launches++;
}
void launch_root_apply(int f, const FrontDev* fr, const double* F, const int* dofs, double* X,
                       int64_t ldx, int nrhs, double* W, const int64_t* woff, cudaStream_t st) {
  k_root_apply<<<1, ST, 0, st>>>(f, fr, F, dofs, X, ldx, nrhs, W, woff);
  g_launches++;
}
void launch_sep_gather(const int* slist, int ns, const SepDev* sp, const int* dofs, double* X,
                       int64_t ldx, int nrhs, const double* W, const int64_t* woff,
                       const FrontDev* fr, cudaStream_t st) {
  if (ns <= 0) return;
  k_sep_gather<<<ns, ST, 0, st>>>(slist, sp, dofs, X, ldx, nrhs, W, woff, fr);
  g_launches++;
}

}  // namespace mfgpu
