// Panel-by-panel partial Cholesky without grid barriers (both precisions).
//
// The reference factors a front's pivot block and forms its Schur complement
// in one dense LU call sequence (src/DE/mf2d.cpp:558-576).  Here, for the
// fronts of one tree level, a W-column panel [Ks, Ks + kb) of every front
// (kb = min(W, n - Ks), W = 64 in FP64, 128 in FP32; every earlier update
// already applied) becomes L in two launches:
//   k_diag_factor  one CTA per front factors the kb x kb diagonal block in
//                  shared memory, 32 columns at a time (a warp's register
//                  Cholesky of the 32 x 32 block with its inverse, the rows
//                  below it by that inverse, the rest of the block by 4 x 4
//                  register tiles), writes L11 back and leaves the inverse of
//                  L11 in the front's scratch slot, K-major;
//   k_panel_trsm   the rows below the block, L21 = A21 L11^{-T}, as one
//                  product with that inverse: 128-row items over a persistent
//                  grid, each CTA a 128 x W tile of A21 and the inverse in
//                  shared memory (K-major, 16-byte vector loads), 8 x (W/16)
//                  outputs per thread in registers.
// The trailing update then follows (k_trail_syrk here, the tensor-core update
// on the mixed path's large levels).  The diagonal block is the only serial
// part and it is factored once, by one CTA; the panel below is plain
// throughput work.  A non-positive pivot records error code 1 (front, column).
#include <algorithm>
#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int kPanThreads = 256;
constexpr int kTrsmRows = 128;            // rows per k_panel_trsm item

template <class T>
__device__ __forceinline__ T rsq(T x);
template <>
__device__ __forceinline__ float rsq<float>(float x) { return rsqrtf(x); }
template <>
__device__ __forceinline__ double rsq<double>(double x) { return rsqrt(x); }

// Shared-memory strides.  Diagonal kernel: row-major W x (W + 1), so that a
// warp reading a column (32 rows, one value each) hits 32 banks.  TRSM
// kernel: K-major rows padded by 16 bytes (vector loads stay aligned).
template <int W>
constexpr int diag_stride() { return W + 1; }
template <class T>
constexpr int vpad() { return 16 / (int)sizeof(T); }
template <class T>
constexpr int xs_stride() { return kTrsmRows + vpad<T>(); }
template <class T, int W>
constexpr int ls_stride() { return W + vpad<T>(); }

template <class T, int W>
constexpr size_t diag_smem() {
  return (size_t)2 * W * diag_stride<W>() * sizeof(T);
}
template <class T, int W>
constexpr size_t trsm_smem() {
  return ((size_t)W * xs_stride<T>() + (size_t)W * ls_stride<T, W>()) * sizeof(T);
}

// Four consecutive values from 16-byte aligned shared memory.
__device__ __forceinline__ void ld4(const float* p, float v[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// One warp factors the jb x jb (jb <= 32) diagonal block at (j0, j0) of Ds
// (row-major, stride S) in place - lane i holds row i in registers, the
// columns are eliminated by shuffles - and writes the inverse of the factor
// to Li (row-major, stride LS; zero above the diagonal and outside jb).
// Returns the first non-positive pivot column of the block, or -1.
template <class T, int S, int LS>
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
    Li[i * LS + lane] = v;
  }
  __syncwarp();
  return bad;
}

// The kb x kb diagonal block of every front's panel, a CTA per front:
// right-looking over 32-column blocks (warp register Cholesky and inverse of
// the block, the rows below it times that inverse by a warp per row, the rest
// of the block by 4 x 4 register tiles), then the inverse of L11 block row by
// block row, V(r, c) = -Li_r sum_{k=c}^{r-1} L(r, k) V(k, c).  Writes L11 into
// the front (lower triangle) and the inverse, K-major (slot[t W + c] =
// Linv(c, t), zero outside the lower kb x kb triangle), into the front's slot.
template <class T, int W>
__global__ void __launch_bounds__(kPanThreads) k_diag_factor(const int* __restrict__ flist,
                                                             const FrontDev* __restrict__ fr,
                                                             T* __restrict__ F, int Ks,
                                                             T* __restrict__ slot, DevError* err) {
  constexpr int S = diag_stride<W>(), NB = W / 32;
  constexpr int ME = NB > 1 ? (NB - 1) * 1024 / kPanThreads : 1;   // inverse entries per thread
  extern __shared__ __align__(16) unsigned char diag_raw[];
  T* As = reinterpret_cast<T*>(diag_raw);   // the block, then L11 (row-major, stride S)
  T* Vs = As + W * S;                       // the inverse of L11 (row-major, stride S)
  __shared__ int badcol;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const FrontDev d = fr[flist[blockIdx.x]];
  if (Ks >= d.n) return;
  T* A = F + d.off;
  const int64_t ld = d.ld;
  const int kb = min(W, d.n - Ks), nb = (kb + 31) / 32;
  for (int idx = tid; idx < W * W; idx += kPanThreads) {
    const int r = idx % W, c = idx / W;
    As[r * S + c] = (r < kb && c <= r) ? A[(Ks + r) + (int64_t)(Ks + c) * ld] : T(0);
    Vs[r * S + c] = T(0);
  }
  if (tid == 0) badcol = -1;
  __syncthreads();
  for (int b = 0; b < nb; b++) {
    const int c0 = 32 * b, jb = min(32, kb - c0), c1 = c0 + jb;
    if (warp == 0) {
      const int bad = warp_chol_inv<T, S, S>(As, c0, jb, Vs + c0 * S + c0);
      if (lane == 0 && bad >= 0 && badcol < 0) badcol = Ks + c0 + bad;
    }
    __syncthreads();
    // rows below block b (jb = 32 whenever there are any): L(r, c0 + c) =
    // sum_t A(r, c0 + t) Linv_b(c, t), a warp per row, lane c
    for (int r = c1 + warp; r < kb; r += kPanThreads / 32) {
      T acc = T(0);
#pragma unroll 8
      for (int t = 0; t < 32; t++) acc += As[r * S + c0 + t] * Vs[(c0 + lane) * S + c0 + t];
      __syncwarp();
      As[r * S + c0 + lane] = acc;
    }
    __syncthreads();
    // the rest of the block: A(r, c) -= sum_t L(r, c0 + t) L(c, c0 + t), c <= r
    const int m4 = (kb - c1 + 3) / 4, ntile = m4 * (m4 + 1) / 2;
    for (int tI = tid; tI < ntile; tI += kPanThreads) {
      int ti = (int)((sqrtf(8.f * (float)tI + 1.f) - 1.f) * 0.5f);   // tile row of lower index tI
      while (ti * (ti + 1) / 2 > tI) ti--;
      while ((ti + 1) * (ti + 2) / 2 <= tI) ti++;
      const int ra = c1 + 4 * ti, ca = c1 + 4 * (tI - ti * (ti + 1) / 2);
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = T(0);
#pragma unroll 4
      for (int t = 0; t < 32; t++) {
        T a[4], bb[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          a[i] = ra + i < kb ? As[(ra + i) * S + c0 + t] : T(0);
          bb[i] = ca + i < kb ? As[(ca + i) * S + c0 + t] : T(0);
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] += a[i] * bb[j];
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (ra + i < kb && ca + j <= ra + i) As[(ra + i) * S + ca + j] -= acc[i][j];
    }
    __syncthreads();
  }
  // the inverse below its diagonal blocks, block row rb at a time
  for (int rb = 1; rb < nb; rb++) {
    const int R0 = 32 * rb, ne = rb * 1024;
    // sum_{k} L(rb, k) V(k, c) into block (rb, c) of Vs: nothing reads that block row yet
#pragma unroll
    for (int q = 0; q < ME; q++) {
      const int e = tid + q * kPanThreads;
      if (e < ne) {
        const int cb = e >> 10, i = (e >> 5) & 31, j = e & 31;
        T acc = T(0);
        for (int k = 32 * cb; k < R0; k++) acc += As[(R0 + i) * S + k] * Vs[k * S + 32 * cb + j];
        Vs[(R0 + i) * S + 32 * cb + j] = acc;
      }
    }
    __syncthreads();
    T v[ME];
#pragma unroll
    for (int q = 0; q < ME; q++) {
      const int e = tid + q * kPanThreads;
      v[q] = T(0);
      if (e < ne) {
        const int cb = e >> 10, i = (e >> 5) & 31, j = e & 31;
        T acc = T(0);
        for (int t = 0; t <= i; t++)
          acc += Vs[(R0 + i) * S + R0 + t] * Vs[(R0 + t) * S + 32 * cb + j];
        v[q] = -acc;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < ME; q++) {
      const int e = tid + q * kPanThreads;
      if (e < ne) Vs[(R0 + ((e >> 5) & 31)) * S + 32 * (e >> 10) + (e & 31)] = v[q];
    }
    __syncthreads();
  }
  if (tid == 0 && badcol >= 0 && atomicCAS(&err->code, 0, 1) == 0) {
    err->front = flist[blockIdx.x];
    err->col = badcol;
  }
  for (int idx = tid; idx < kb * kb; idx += kPanThreads) {
    const int r = idx % kb, c = idx / kb;
    if (c <= r) A[(Ks + r) + (int64_t)(Ks + c) * ld] = As[r * S + c];
  }
  T* Lt = slot + (int64_t)blockIdx.x * W * W;
  for (int idx = tid; idx < W * W; idx += kPanThreads) Lt[idx] = Vs[(idx % W) * S + idx / W];
}

// The rows below the diagonal block, L21 = A21 L11^{-T} = A21 Linv^T, over a
// persistent grid.  Items are 128-row blocks of every front's rows [Ks + kb,
// N), listed front by front.  A CTA holds the tile K-major (Xs[t][r]) and the
// front's inverse K-major (Ls[t][c] = Linv(c, t), loaded once per front it
// visits); thread (tx, ty) accumulates rows 4 ty .. 4 ty + 3 and 64 + the
// same, columns tx + 16 j (+ 64 h) in registers.  Linv(c, t) = 0 for t > c, so
// past t = 64 h only the column groups from h on take part.  The result goes
// through shared memory (row-major, stride W + 1) for coalesced stores.
template <class T, int W>
__global__ void __launch_bounds__(kPanThreads) k_panel_trsm(const int* __restrict__ flist, int nf,
                                                            const FrontDev* __restrict__ fr,
                                                            T* __restrict__ F, int Ks,
                                                            const T* __restrict__ slot) {
  constexpr int XS = xs_stride<T>(), LS = ls_stride<T, W>(), CG = W / 64, RS = W + 1;
  static_assert(kTrsmRows * RS <= W * XS, "result tile must fit the input tile");
  extern __shared__ __align__(16) unsigned char trsm_raw[];
  T* Xs = reinterpret_cast<T*>(trsm_raw);   // the tile (K-major), then the result (row-major)
  T* Ls = Xs + W * XS;                       // the inverse, K-major
  __shared__ int pre[kMaxPanelFronts + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int i = tid; i < nf; i += kPanThreads) {
    const FrontDev d = fr[flist[i]];
    pre[i + 1] = Ks < d.n ? (d.N - Ks - min(W, d.n - Ks) + kTrsmRows - 1) / kTrsmRows : 0;
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
    const int i = lo;
    const FrontDev d = fr[flist[i]];
    T* A = F + d.off;
    const int64_t ld = d.ld;
    const int kb = min(W, d.n - Ks);
    const int r0 = Ks + kb + (item - pre[i]) * kTrsmRows, rows = min(kTrsmRows, d.N - r0);
    __syncthreads();                         // the previous item's result has been stored
    if (i != cur) {
      cur = i;
      const T* Lt = slot + (int64_t)i * W * W;
      for (int idx = tid; idx < W * W; idx += kPanThreads) Ls[(idx / W) * LS + idx % W] = Lt[idx];
    }
    for (int idx = tid; idx < W * kTrsmRows; idx += kPanThreads) {
      const int r = idx % kTrsmRows, t = idx / kTrsmRows;
      Xs[t * XS + r] = (r < rows && t < kb) ? A[(r0 + r) + (int64_t)(Ks + t) * ld] : T(0);
    }
    __syncthreads();
    T acc[8][4 * CG];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
      for (int c = 0; c < 4 * CG; c++) acc[a][c] = T(0);
#pragma unroll
    for (int hs = 0; hs < CG; hs++) {
      const int tend = min(kb, 64 * hs + 64);
      for (int t = 64 * hs; t < tend; t++) {
        T a[8], b[4 * CG];
        ld4(Xs + t * XS + 4 * ty, a);
        ld4(Xs + t * XS + 64 + 4 * ty, a + 4);
#pragma unroll
        for (int h = hs; h < CG; h++)
#pragma unroll
          for (int j = 0; j < 4; j++) b[4 * h + j] = Ls[t * LS + 64 * h + tx + 16 * j];
#pragma unroll
        for (int r = 0; r < 8; r++)
#pragma unroll
          for (int h = hs; h < CG; h++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[r][4 * h + j] = fma(a[r], b[4 * h + j], acc[r][4 * h + j]);
      }
    }
    __syncthreads();                         // every read of the tile is done
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
      for (int h = 0; h < CG; h++)
#pragma unroll
        for (int j = 0; j < 4; j++)
          Xs[(64 * (r >> 2) + 4 * ty + (r & 3)) * RS + 64 * h + tx + 16 * j] = acc[r][4 * h + j];
    __syncthreads();
    for (int idx = tid; idx < kb * kTrsmRows; idx += kPanThreads) {
      const int r = idx % kTrsmRows, c = idx / kTrsmRows;
      if (r < rows) A[(r0 + r) + (int64_t)(Ks + c) * ld] = Xs[r * RS + c];
    }
  }
}

template <class T, int W>
cudaError_t launchPanel(const int* flist, int nf, const FrontDev* fr, T* F, int Ks, T* slot,
                        DevError* err, cudaStream_t st) {
  static const int grid = []() {   // thread-safe one-time set-up: every resident CTA
    int dev = 0, n = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_diag_factor<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)diag_smem<T, W>());
    cudaFuncSetAttribute(k_panel_trsm<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)trsm_smem<T, W>());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_panel_trsm<T, W>, kPanThreads,
                                                  trsm_smem<T, W>());
    return n * std::max(1, per);
  }();
  k_diag_factor<T, W><<<nf, kPanThreads, diag_smem<T, W>(), st>>>(flist, fr, F, Ks, slot, err);
  k_panel_trsm<T, W><<<grid, kPanThreads, trsm_smem<T, W>(), st>>>(flist, nf, fr, F, Ks, slot);
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
  return launchPanel<float, kPanelW32>(flist, nf, fr, F, Ks, dslot, err, st);
}
template <>
cudaError_t launch_subpanel<double>(const int* flist, int nf, const FrontDev* fr, double* F, int Ks,
                                    int w, double* dslot, DevError* err, cudaStream_t st) {
  if (nf <= 0) return cudaSuccess;
  if (nf > kMaxPanelFronts || w != kPanelW64 || !dslot) return cudaErrorInvalidValue;
  return launchPanel<double, kPanelW64>(flist, nf, fr, F, Ks, dslot, err, st);
}

}  // namespace mfgpu
