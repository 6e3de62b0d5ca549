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
#include <atomic>
#include <cstdio>

#include "device.cuh"

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
// Panel step k of the right-looking partial Cholesky, for all fronts of a list.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void report(DevError* err, int code, int front, int col) {
  if (atomicCAS(&err->code, 0, code) == 0) {
    err->front = front;
    err->col = col;
  }
}

__global__ void __launch_bounds__(32) k_potrf(const int* __restrict__ flist,
                                              const FrontDev* __restrict__ fr,
                                              double* __restrict__ F, int k, DevError* err) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  if (k >= d.n) return;
  const int kb = min(kPanel, d.n - k);
  __shared__ double D[kPanel][kPanel + 1];
  double* A = F + d.off + k + (int64_t)k * d.ld;
  const int lane = threadIdx.x;
  for (int j = 0; j < kb; j++)
    if (lane < kb && lane >= j) D[lane][j] = A[lane + (int64_t)j * d.ld];
  __syncwarp();
  bool bad = false;
  for (int j = 0; j < kb; j++) {
    double djj = D[j][j];
    if (!(djj > 0.0)) {               // non-positive or NaN pivot: not SPD
      if (lane == 0 && !bad) report(err, 1, f, k + j);
      bad = true;
      djj = 1.0;
    }
    const double s = sqrt(djj);
    __syncwarp();
    if (lane == j) D[j][j] = s;
    if (lane > j && lane < kb) D[lane][j] = D[lane][j] / s;
    __syncwarp();
    if (lane > j && lane < kb) {
      const double lij = D[lane][j];
      for (int l = j + 1; l <= lane; l++) D[lane][l] -= lij * D[l][j];
    }
    __syncwarp();
  }
  for (int j = 0; j < kb; j++)
    if (lane < kb && lane >= j) A[lane + (int64_t)j * d.ld] = D[lane][j];
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
  double* A = F + d.off;
  for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
    int i = idx % kb, j = idx / kb;
    if (i >= j) L[i][j] = A[(k + i) + (int64_t)(k + j) * d.ld];
  }
  __syncthreads();
  const int r = k + kb + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.N) return;
  double x[kPanel];
#pragma unroll
  for (int t = 0; t < kPanel; t++) x[t] = t < kb ? A[r + (int64_t)(k + t) * d.ld] : 0.0;
#pragma unroll
  for (int j = 0; j < kPanel; j++) {
    if (j < kb) {
      double s = x[j];
#pragma unroll
      for (int t = 0; t < j; t++) s -= x[t] * L[j][t];
      x[j] = s / L[j][j];
    }
  }
#pragma unroll
  for (int t = 0; t < kPanel; t++)
    if (t < kb) A[r + (int64_t)(k + t) * d.ld] = x[t];
}

// Trailing update C(r, c) -= sum_t X(r, t) X(c, t), r >= c, over [k+kb, N)^2.
constexpr int UT = 64;
__global__ void __launch_bounds__(256) k_syrk(const int* __restrict__ flist,
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
  const int t = blockIdx.x;
  if (t >= T * (T + 1) / 2) return;
  int I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while (I * (I + 1) / 2 > t) I--;
  while ((I + 1) * (I + 2) / 2 <= t) I++;
  const int J = t - I * (I + 1) / 2;
  __shared__ double Xa[kPanel][UT + 1];
  __shared__ double Xb[kPanel][UT + 1];
  double* A = F + d.off;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < UT * kPanel; idx += 256) {
    int i = idx % UT, tt = idx / UT;
    int ra = r0 + I * UT + i, rb = r0 + J * UT + i;
    bool ok = tt < kb;
    Xa[tt][i] = (ok && ra < d.N) ? A[ra + (int64_t)(k + tt) * d.ld] : 0.0;
    Xb[tt][i] = (ok && rb < d.N) ? A[rb + (int64_t)(k + tt) * d.ld] : 0.0;
  }
  __syncthreads();
  const int tx = tid % 16, ty = tid / 16;
  double acc[4][4] = {};
  for (int tt = 0; tt < kb; tt++) {
    double a[4], b[4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      a[p] = Xa[tt][tx + 16 * p];
      b[p] = Xb[tt][ty + 16 * p];
    }
#pragma unroll
    for (int p = 0; p < 4; p++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[p][q] = fma(a[p], b[q], acc[p][q]);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = r0 + J * UT + ty + 16 * q;
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const int r = r0 + I * UT + tx + 16 * p;
      if (r < d.N && c < d.N && r >= c) A[r + (int64_t)c * d.ld] -= acc[p][q];
    }
  }
}

// ---------------------------------------------------------------------------
// Solve / apply sweeps.  One CTA per front; W is the front's workspace (N x nrhs,
// ld N) inside a shared buffer.
// ---------------------------------------------------------------------------
constexpr int ST = 256;

// Forward solve with the front's first n columns, right-looking over 32-column
// blocks.  On exit W[0,n) = L11^{-1} b_piv and W[n,N) = -L21 W[0,n).
__device__ void front_forward(const FrontDev& d, const double* __restrict__ A, double* W,
                              int nrhs) {
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  for (int k = 0; k < n; k += kPanel) {
    const int kb = min(kPanel, n - k);
    if (tid < nrhs) {
      double* w = W + (int64_t)tid * N;
      for (int j = 0; j < kb; j++) {
        double s = w[k + j];
        for (int t = 0; t < j; t++) s -= A[(k + j) + (int64_t)(k + t) * ld] * w[k + t];
        w[k + j] = s / A[(k + j) + (int64_t)(k + j) * ld];
      }
    }
    __syncthreads();
    const int rows = N - k - kb;
    for (int idx = tid; idx < rows * nrhs; idx += blockDim.x) {
      const int r = k + kb + idx % rows, c = idx / rows;
      const double* w = W + (int64_t)c * N;
      double s = 0.0;
      for (int t = 0; t < kb; t++) s += A[r + (int64_t)(k + t) * ld] * w[k + t];
      W[r + (int64_t)c * N] -= s;
    }
    __syncthreads();
  }
}

// Backward solve: W[0,n) <- L11^{-T} (W[0,n) - L21^T W[n,N)).
__device__ void front_backward(const FrontDev& d, const double* __restrict__ A, double* W,
                               int nrhs) {
  const int N = d.N, n = d.n, ld = d.ld, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  __shared__ double part[kPanel * 16];
  const int nblk = (n + kPanel - 1) / kPanel;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int k = bk * kPanel;
    const int kb = min(kPanel, n - k);
    // s(j, c) = sum_{r >= k+kb} L(r, k+j) W(r, c)
    for (int jc = warp; jc < kb * nrhs; jc += nw) {
      const int j = jc % kb, c = jc / kb;
      const double* w = W + (int64_t)c * N;
      double s = 0.0;
      for (int r = k + kb + lane; r < N; r += 32) s += A[r + (int64_t)(k + j) * ld] * w[r];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) part[jc] = s;
    }
    __syncthreads();
    if (tid < nrhs) {
      double* w = W + (int64_t)tid * N;
      for (int j = kb - 1; j >= 0; j--) {
        double s = w[k + j] - part[j + tid * kb];
        for (int t = j + 1; t < kb; t++) s -= A[(k + t) + (int64_t)(k + j) * ld] * w[k + t];
        w[k + j] = s / A[(k + j) + (int64_t)(k + j) * ld];
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(ST) k_solve_fwd(const int* __restrict__ flist,
                                                  const FrontDev* __restrict__ fr,
                                                  const double* __restrict__ F,
                                                  const int* __restrict__ dofs, double* X,
                                                  int64_t ldx, int nrhs, double* Wb,
                                                  const int64_t* __restrict__ woff) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = i < d.n ? X[dl[i] + (int64_t)c * ldx] : 0.0;
  }
  __syncthreads();
  front_forward(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

__global__ void __launch_bounds__(ST) k_solve_bwd(const int* __restrict__ flist,
                                                  const FrontDev* __restrict__ fr,
                                                  const double* __restrict__ F,
                                                  const int* __restrict__ dofs, double* X,
                                                  int64_t ldx, int nrhs, double* Wb,
                                                  const int64_t* __restrict__ woff) {
  const int f = flist[blockIdx.x];
  const FrontDev d = fr[f];
  double* W = Wb + woff[f] * nrhs;
  const int* dl = dofs + d.dof_off;
  for (int idx = threadIdx.x; idx < d.N * nrhs; idx += blockDim.x) {
    const int i = idx % d.N, c = idx / d.N;
    W[idx] = X[dl[i] + (int64_t)c * ldx];
  }
  __syncthreads();
  front_backward(d, F + d.off, W, nrhs);
  for (int idx = threadIdx.x; idx < d.n * nrhs; idx += blockDim.x) {
    const int i = idx % d.n, c = idx / d.n;
    X[dl[i] + (int64_t)c * ldx] = W[i + (int64_t)c * d.N];
  }
}

__global__ void __launch_bounds__(ST) k_root_solve(int f, const FrontDev* __restrict__ fr,
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
  front_forward(d, F + d.off, W, nrhs);
  front_backward(d, F + d.off, W, nrhs);
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
  k_syrk<<<dim3(T * (T + 1) / 2, nf), 256, 0, st>>>(flist, fr, F, k);
  g_launches++;
}

long long launches_total() { return g_launches.load(); }

void launch_solve_fwd(const int* flist, int nf, const FrontDev* fr, const double* F,
                      const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                      const int64_t* woff, cudaStream_t st) {
  if (nf <= 0) return;
  k_solve_fwd<<<nf, ST, 0, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff);
  g_launches++;
}
void launch_solve_bwd(const int* flist, int nf, const FrontDev* fr, const double* F,
                      const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                      const int64_t* woff, cudaStream_t st) {
  if (nf <= 0) return;
  k_solve_bwd<<<nf, ST, 0, st>>>(flist, fr, F, dofs, X, ldx, nrhs, W, woff);
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
void launch_root_solve(int f, const FrontDev* fr, const double* F, const int* dofs, double* X,
                       int64_t ldx, int nrhs, double* W, const int64_t* woff, cudaStream_t st) {
  k_root_solve<<<1, ST, 0, st>>>(f, fr, F, dofs, X, ldx, nrhs, W, woff);
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
