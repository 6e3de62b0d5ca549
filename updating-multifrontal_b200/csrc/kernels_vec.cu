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

// Deterministic, segmented dot products.  The vector is a concatenation of
// segments (the problems of a batch; one segment otherwise); each segment is
// cut into chunks of kDotChunk elements starting at the segment's first row,
// each chunk reduced by a fixed tree, and a segment's chunk sums added in
// order.  A segment's result therefore depends only on its own data.
constexpr int kDotChunk = 8192;

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

// chunk_row[k] = first row of chunk k; chunk_row[nchunks] = n.
__global__ void k_dot_part(const double* __restrict__ x, int64_t ldx, const double* __restrict__ y,
                           int64_t ldy, const int* __restrict__ chunk_row, int nchunks,
                           double* __restrict__ part) {
  const int k = blockIdx.x, c = blockIdx.y;
  const int lo = chunk_row[k], hi = chunk_row[k + 1];
  const double* xc = x + c * ldx;
  const double* yc = y + c * ldy;
  double s = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += VT) s = fma(xc[i], yc[i], s);
  s = block_sum(s);
  if (threadIdx.x == 0) part[(int64_t)c * nchunks + k] = s;
}

// out[seg + nseg * c] = sum of the segment's chunk partials, in order.
__global__ void k_dot_final(const double* __restrict__ part, const int* __restrict__ seg_chunk,
                            int nseg, int nchunks, double* __restrict__ out) {
  const int g = blockIdx.x, c = blockIdx.y;
  const int lo = seg_chunk[g], hi = seg_chunk[g + 1];
  double s = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += VT) s += part[(int64_t)c * nchunks + i];
  s = block_sum(s);
  if (threadIdx.x == 0) out[g + nseg * c] = s;
}

__device__ __forceinline__ int seg_of(const int* __restrict__ seg_row, int nseg, int i) {
  int lo = 0, hi = nseg - 1;   // largest g with seg_row[g] <= i
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg_row[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
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

// x += a p ; r -= a q with a = rz / pq of the row's (segment, column), for
// active (segment, column) pairs.
__global__ void k_pcg_xr(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                         const double* __restrict__ q, int64_t ld, int n,
                         const double* __restrict__ rz, const double* __restrict__ pq,
                         const int* __restrict__ active, const int* __restrict__ seg_row, int nseg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n) return;
  const int g = seg_of(seg_row, nseg, i) + nseg * c;
  if (!active[g]) return;
  const double a = rz[g] / pq[g];
  x[i + c * ld] = fma(a, p[i + c * ld], x[i + c * ld]);
  r[i + c * ld] = fma(-a, q[i + c * ld], r[i + c * ld]);
}

// p = z + b p with b = rz_new / rz_old of the row's (segment, column) (first
// iteration: p = z).
__global__ void k_pcg_p(double* __restrict__ p, const double* __restrict__ z, int64_t ld, int n,
                        const double* __restrict__ rz_new, const double* __restrict__ rz_old,
                        const int* __restrict__ active, int first, const int* __restrict__ seg_row,
                        int nseg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= n) return;
  const int g = seg_of(seg_row, nseg, i) + nseg * c;
  if (!active[g]) return;
  const double b = first ? 0.0 : rz_new[g] / rz_old[g];
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

void dot_plan(const std::vector<int64_t>& seg_row, std::vector<int>& chunk_row,
              std::vector<int>& seg_chunk) {
  chunk_row.clear();
  seg_chunk.assign(1, 0);
  for (size_t g = 0; g + 1 < seg_row.size(); g++) {
    for (int64_t r = seg_row[g]; r < seg_row[g + 1]; r += kDotChunk) chunk_row.push_back((int)r);
    seg_chunk.push_back((int)chunk_row.size());
  }
  chunk_row.push_back((int)seg_row.back());
}

void launch_dot(const double* x, int64_t ldx, const double* y, int64_t ldy, int nrhs,
                const int* chunk_row, int nchunks, const int* seg_chunk, int nseg, double* part,
                double* out, cudaStream_t st) {
  k_dot_part<<<dim3(nchunks, nrhs), VT, 0, st>>>(x, ldx, y, ldy, chunk_row, nchunks, part);
  k_dot_final<<<dim3(nseg, nrhs), VT, 0, st>>>(part, seg_chunk, nseg, nchunks, out);
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
                   int nrhs, const double* rz, const double* pq, const int* active,
                   const int* seg_row, int nseg, cudaStream_t st) {
  k_pcg_xr<<<vgrid(n, nrhs), VT, 0, st>>>(x, r, p, q, ld, n, rz, pq, active, seg_row, nseg);
  g_launches++;
}

void launch_pcg_p(double* p, const double* z, int64_t ld, int n, int nrhs, const double* rz_new,
                  const double* rz_old, const int* active, int first, const int* seg_row, int nseg,
                  cudaStream_t st) {
  k_pcg_p<<<vgrid(n, nrhs), VT, 0, st>>>(p, z, ld, n, rz_new, rz_old, active, first, seg_row, nseg);
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
