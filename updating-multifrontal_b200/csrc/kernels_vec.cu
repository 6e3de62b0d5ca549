// Vector kernels of the mixed-precision solve: FP64 sparse matrix-vector
// products (the refinement residual r = b - A x), deterministic dot products,
// the preconditioned conjugate-gradient updates, and the conversions between
// the FP64 iterate and the FP32 factorization's scaled variables.
//
// All multi-column kernels take column-major n x nrhs blocks with a leading
// dimension; column c of a block lives at base + c * ld.
#include <atomic>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int VT = 256;

// s_i = 1 / sqrt(A_ii): the symmetric diagonal scaling of the FP32 factor;
// is_i = 1 / s_i.
__global__ void k_diag_scale(const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ va, int n, double* __restrict__ s,
                             double* __restrict__ is) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; p++)
    if (ci[p] == i) d = va[p];
  const double r = d > 0.0 ? sqrt(d) : 1.0;
  s[i] = 1.0 / r;
  is[i] = r;
}

// y = A x, one thread per row and column (rows of a 5/7-point stencil are short).
__global__ void k_spmv(const int* __restrict__ rp, const int* __restrict__ ci,
                       const double* __restrict__ va, int n, const double* __restrict__ x,
                       int64_t ldx, double* __restrict__ y, int64_t ldy, int nrhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n || c >= nrhs) return;
  const double* xc = x + c * ldx;
  double s = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; p++) s = fma(va[p], xc[ci[p]], s);
  y[i + c * ldy] = s;
}

// y = b - A x
__global__ void k_residual(const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ va, int n, const double* __restrict__ b,
                           int64_t ldb, const double* __restrict__ x, int64_t ldx,
                           double* __restrict__ r, int64_t ldr, int nrhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n || c >= nrhs) return;
  const double* xc = x + c * ldx;
  double s = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; p++) s = fma(va[p], xc[ci[p]], s);
  r[i + c * ldr] = b[i + c * ldb] - s;
}

// Deterministic dot products: fixed partition into kDotBlocks chunks, fixed
// reduction tree in each, partials summed in order by one block per column.
constexpr int kDotBlocks = 256;

__device__ double block_sum(double v) {
  __shared__ double red[VT / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < VT / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;   // valid in thread 0
}

__global__ void k_dot_part(const double* __restrict__ x, int64_t ldx, const double* __restrict__ y,
                           int64_t ldy, int n, double* __restrict__ part) {
  const int c = blockIdx.y;
  const int chunk = (n + kDotBlocks - 1) / kDotBlocks;
  const int lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
  const double* xc = x + c * ldx;
  const double* yc = y + c * ldy;
  double s = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += VT) s = fma(xc[i], yc[i], s);
  s = block_sum(s);
  if (threadIdx.x == 0) part[c * kDotBlocks + blockIdx.x] = s;
}

__global__ void k_dot_final(const double* __restrict__ part, double* __restrict__ out) {
  const int c = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < kDotBlocks; i += VT) s += part[c * kDotBlocks + i];
  s = block_sum(s);
  if (threadIdx.x == 0) out[c] = s;
}

// dst(T) = s .* src(double)   (s may be null)
template <class T>
__global__ void k_scale_to(const double* __restrict__ src, int64_t lds, T* __restrict__ dst,
                           int64_t ldd, const double* __restrict__ s, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n) return;
  const double v = src[i + c * lds];
  dst[i + c * ldd] = (T)(s ? s[i] * v : v);
}

// dst(double) = s .* src(T)   (s may be null)
template <class T>
__global__ void k_scale_from(const T* __restrict__ src, int64_t lds, double* __restrict__ dst,
                             int64_t ldd, const double* __restrict__ s, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n) return;
  const double v = (double)src[i + c * lds];
  dst[i + c * ldd] = s ? s[i] * v : v;
}

// x_c += a_c p_c ; r_c -= a_c q_c with a_c = rz_c / pq_c, for active columns.
__global__ void k_pcg_xr(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                         const double* __restrict__ q, int64_t ld, int n,
                         const double* __restrict__ rz, const double* __restrict__ pq,
                         const int* __restrict__ active) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n || !active[c]) return;
  const double a = rz[c] / pq[c];
  x[i + c * ld] = fma(a, p[i + c * ld], x[i + c * ld]);
  r[i + c * ld] = fma(-a, q[i + c * ld], r[i + c * ld]);
}

// p_c = z_c + b_c p_c with b_c = rz_new_c / rz_old_c (first iteration: p = z).
__global__ void k_pcg_p(double* __restrict__ p, const double* __restrict__ z, int64_t ld, int n,
                        const double* __restrict__ rz_new, const double* __restrict__ rz_old,
                        const int* __restrict__ active, int first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n || !active[c]) return;
  const double b = first ? 0.0 : rz_new[c] / rz_old[c];
  p[i + c * ld] = fma(b, p[i + c * ld], z[i + c * ld]);
}

inline dim3 vgrid(int n, int nrhs) { return dim3((n + VT - 1) / VT, nrhs); }

}  // namespace

void launch_diag_scale(const int* rp, const int* ci, const double* va, int n, double* s,
                       double* is, cudaStream_t st) {
  k_diag_scale<<<(n + VT - 1) / VT, VT, 0, st>>>(rp, ci, va, n, s, is);
  g_launches++;
}

void launch_spmv(const int* rp, const int* ci, const double* va, int n, const double* x, int64_t ldx,
                 double* y, int64_t ldy, int nrhs, cudaStream_t st) {
  k_spmv<<<vgrid(n, nrhs), VT, 0, st>>>(rp, ci, va, n, x, ldx, y, ldy, nrhs);
  g_launches++;
}

void launch_residual(const int* rp, const int* ci, const double* va, int n, const double* b,
                     int64_t ldb, const double* x, int64_t ldx, double* r, int64_t ldr, int nrhs,
                     cudaStream_t st) {
  k_residual<<<vgrid(n, nrhs), VT, 0, st>>>(rp, ci, va, n, b, ldb, x, ldx, r, ldr, nrhs);
  g_launches++;
}

size_t dot_scratch_elems(int nrhs) { return (size_t)kDotBlocks * nrhs; }

void launch_dot(const double* x, int64_t ldx, const double* y, int64_t ldy, int n, int nrhs,
                double* part, double* out, cudaStream_t st) {
  k_dot_part<<<dim3(kDotBlocks, nrhs), VT, 0, st>>>(x, ldx, y, ldy, n, part);
  k_dot_final<<<nrhs, VT, 0, st>>>(part, out);
  g_launches += 2;
}

template <class T>
void launch_scale_to(const double* src, int64_t lds, T* dst, int64_t ldd, const double* s, int n,
                     int nrhs, cudaStream_t st) {
  k_scale_to<T><<<vgrid(n, nrhs), VT, 0, st>>>(src, lds, dst, ldd, s, n);
  g_launches++;
}

template <class T>
void launch_scale_from(const T* src, int64_t lds, double* dst, int64_t ldd, const double* s, int n,
                       int nrhs, cudaStream_t st) {
  k_scale_from<T><<<vgrid(n, nrhs), VT, 0, st>>>(src, lds, dst, ldd, s, n);
  g_launches++;
}

void launch_pcg_xr(double* x, double* r, const double* p, const double* q, int64_t ld, int n,
                   int nrhs, const double* rz, const double* pq, const int* active, cudaStream_t st) {
  k_pcg_xr<<<vgrid(n, nrhs), VT, 0, st>>>(x, r, p, q, ld, n, rz, pq, active);
  g_launches++;
}

void launch_pcg_p(double* p, const double* z, int64_t ld, int n, int nrhs, const double* rz_new,
                  const double* rz_old, const int* active, int first, cudaStream_t st) {
  k_pcg_p<<<vgrid(n, nrhs), VT, 0, st>>>(p, z, ld, n, rz_new, rz_old, active, first);
  g_launches++;
}

template void launch_scale_to<float>(const double*, int64_t, float*, int64_t, const double*, int, int,
                                     cudaStream_t);
template void launch_scale_to<double>(const double*, int64_t, double*, int64_t, const double*, int,
                                      int, cudaStream_t);
template void launch_scale_from<float>(const float*, int64_t, double*, int64_t, const double*, int,
                                       int, cudaStream_t);
template void launch_scale_from<double>(const double*, int64_t, double*, int64_t, const double*, int,
                                        int, cudaStream_t);

}  // namespace mfgpu
