// Stencil assembly on the device: CSR values of the variable-coefficient
// 5-point (2D) / 7-point (3D) Laplacian from the node coefficient array, and
// detection of the rows a coefficient change modifies.
//
// Restates the reference fixture test_include/DE/buildLaplacian.hpp:10-132
// (2D) and :244-391 (3D) for separator width 1: a face coefficient is
// ahalf = 0.5 * (a[neighbour] + a[self]); the entry towards a neighbour is
// (-1 * ahalf) / h^2 and the diagonal is
// ((0 - (-1 * (ah_x- + ah_x+)) / hx^2) - (-1 * (ah_y- + ah_y+)) / hy^2) [- z term].
// Every value comes from the same sequence of IEEE double operations
// (explicit round-to-nearest intrinsics, so nothing is contracted) and equals
// the fixture's bit for bit.  Entries of a row are in ascending column order:
// z-, y-, x-, self, x+, y+, z+ (2D drops z), present only inside the grid.
//
// Coefficients: (Nx+2) x (Ny+2) [x (Nz+2)] doubles, C order with the x index
// slowest (the fixture's a[i][j][k]); cell (i, j, k) of the grid is node
// (i+1, j+1, k+1).  DOF id = i + j*Nx + k*Nx*Ny.
#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

struct Geo {
  int dim, nx, ny, nz;
  double hh[3];
};

__device__ __forceinline__ double coef(const double* __restrict__ a, const Geo& g, int i, int j,
                                       int k) {   // node indices
  if (g.dim == 2) return a[(int64_t)i * (g.ny + 2) + j];
  return a[((int64_t)i * (g.ny + 2) + j) * (g.nz + 2) + k];
}

__device__ __forceinline__ double ahalf(double x, double y) {
  return __dmul_rn(0.5, __dadd_rn(x, y));
}

__device__ __forceinline__ double offdiag(double ah, double hh) {
  return __ddiv_rn(__dmul_rn(-1.0, ah), hh);
}

// Values of the row of cell (i, j, k) into v[0 .. count); returns count.
__device__ int row_values(const double* __restrict__ a, const Geo& g, int i, int j, int k,
                          double (&v)[7]) {
  const int I = i + 1, J = j + 1, K = g.dim == 3 ? k + 1 : 0;
  const double self = coef(a, g, I, J, K);
  const double xm = ahalf(coef(a, g, I - 1, J, K), self), xp = ahalf(coef(a, g, I + 1, J, K), self);
  const double ym = ahalf(coef(a, g, I, J - 1, K), self), yp = ahalf(coef(a, g, I, J + 1, K), self);
  double zm = 0.0, zp = 0.0;
  if (g.dim == 3) {
    zm = ahalf(coef(a, g, I, J, K - 1), self);
    zp = ahalf(coef(a, g, I, J, K + 1), self);
  }
  double d = 0.0;
  d = __dsub_rn(d, __ddiv_rn(__dmul_rn(-1.0, __dadd_rn(xm, xp)), g.hh[0]));
  d = __dsub_rn(d, __ddiv_rn(__dmul_rn(-1.0, __dadd_rn(ym, yp)), g.hh[1]));
  if (g.dim == 3) d = __dsub_rn(d, __ddiv_rn(__dmul_rn(-1.0, __dadd_rn(zm, zp)), g.hh[2]));
  int c = 0;
  if (g.dim == 3 && k > 0) v[c++] = offdiag(zm, g.hh[2]);
  if (j > 0) v[c++] = offdiag(ym, g.hh[1]);
  if (i > 0) v[c++] = offdiag(xm, g.hh[0]);
  v[c++] = d;
  if (i < g.nx - 1) v[c++] = offdiag(xp, g.hh[0]);
  if (j < g.ny - 1) v[c++] = offdiag(yp, g.hh[1]);
  if (g.dim == 3 && k < g.nz - 1) v[c++] = offdiag(zp, g.hh[2]);
  return c;
}

// Rows of the cells in the box [lo, lo + b) of the grid: recompute the values;
// with `flag`, record whether a row's values changed.
__global__ void k_stencil_rows(const double* __restrict__ a, Geo g, const int* __restrict__ rp,
                               double* __restrict__ val, int lo0, int lo1, int lo2, int bx, int by,
                               int bz, int* __restrict__ flag) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)bx * by * bz) return;
  const int i = lo0 + (int)(t % bx), j = lo1 + (int)((t / bx) % by);
  const int k = lo2 + (int)(t / ((int64_t)bx * by));
  const int64_t row = i + (int64_t)j * g.nx + (int64_t)k * g.nx * g.ny;
  double v[7];
  const int c = row_values(a, g, i, j, k, v);
  const int64_t p0 = rp[row];
  int changed = 0;
  for (int e = 0; e < c; e++) {
    changed |= (val[p0 + e] != v[e]);
    val[p0 + e] = v[e];
  }
  if (flag) flag[row] = changed;
}

__global__ void k_collect(const int* __restrict__ flag, int lo0, int lo1, int lo2, int bx, int by,
                          int bz, int nx, int ny, int* __restrict__ out, int cap,
                          int* __restrict__ count) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)bx * by * bz) return;
  const int i = lo0 + (int)(t % bx), j = lo1 + (int)((t / bx) % by);
  const int k = lo2 + (int)(t / ((int64_t)bx * by));
  const int64_t row = i + (int64_t)j * nx + (int64_t)k * nx * ny;
  if (flag[row]) {
    const int slot = atomicAdd(count, 1);
    if (slot < cap) out[slot] = (int)row;
  }
}

// Coefficients of the cells [lo, hi) multiplied by `factor` (node = cell + 1).
__global__ void k_scale_box(double* __restrict__ a, int dim, int ny, int nz, int lo0, int lo1,
                            int lo2, int bx, int by, int bz, double factor) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)bx * by * bz) return;
  const int i = lo0 + (int)(t % bx) + 1, j = lo1 + (int)((t / bx) % by) + 1;
  const int k = lo2 + (int)(t / ((int64_t)bx * by)) + 1;
  const int64_t idx = dim == 2 ? (int64_t)i * (ny + 2) + j : ((int64_t)i * (ny + 2) + j) * (nz + 2) + k;
  a[idx] = __dmul_rn(a[idx], factor);
}

}  // namespace

cudaError_t launch_scale_box(int dim, int ny, int nz, const int lo[3], const int hi[3], double factor,
                             double* a, cudaStream_t st) {
  const int bx = hi[0] - lo[0], by = hi[1] - lo[1], bz = dim == 3 ? hi[2] - lo[2] : 1;
  if (bx <= 0 || by <= 0 || bz <= 0) return cudaSuccess;
  const int64_t cells = (int64_t)bx * by * bz;
  k_scale_box<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(a, dim, ny, nz, lo[0], lo[1],
                                                              dim == 3 ? lo[2] : 0, bx, by, bz,
                                                              factor);
  g_launches++;
  return cudaGetLastError();
}

cudaError_t launch_stencil_rows(int dim, int nx, int ny, int nz, const double h[3], const double* a,
                                const int* rp, double* val, const int lo[3], const int hi[3],
                                int* flag, cudaStream_t st) {
  const Geo g{dim, nx, ny, dim == 3 ? nz : 1, {h[0] * h[0], h[1] * h[1], h[2] * h[2]}};
  const int bx = hi[0] - lo[0], by = hi[1] - lo[1], bz = dim == 3 ? hi[2] - lo[2] : 1;
  if (bx <= 0 || by <= 0 || bz <= 0) return cudaSuccess;
  const int64_t cells = (int64_t)bx * by * bz;
  k_stencil_rows<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(
      a, g, rp, val, lo[0], lo[1], dim == 3 ? lo[2] : 0, bx, by, bz, flag);
  g_launches++;
  return cudaGetLastError();
}

cudaError_t launch_collect_rows(int dim, int nx, int ny, const int lo[3], const int hi[3],
                                const int* flag, int* out, int cap, int* count, cudaStream_t st) {
  const int bx = hi[0] - lo[0], by = hi[1] - lo[1], bz = dim == 3 ? hi[2] - lo[2] : 1;
  if (bx <= 0 || by <= 0 || bz <= 0) return cudaSuccess;
  const int64_t cells = (int64_t)bx * by * bz;
  k_collect<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(
      flag, lo[0], lo[1], dim == 3 ? lo[2] : 0, bx, by, bz, nx, ny, out, cap, count);
  g_launches++;
  return cudaGetLastError();
}

}  // namespace mfgpu
