// Panel-by-panel partial Cholesky without grid barriers (both precisions).
//
// The reference factors a front's pivot block and forms its Schur complement
// in one dense LU call sequence (src/DE/mf2d.cpp:558-576).  Here, for the
// fronts of one tree level, a W-column panel [Ks, Ks + kb) of every front
// (kb = min(W, n - Ks), W = 64 in FP64, 128 in FP32; every earlier update
// already applied) becomes L in two launches:
//   k_diag_factor  one CTA per front factors the kb x kb diagonal block in
//                  shared memory, 32 columns at a time (a warp's register
//                  Cholesky and inverse of the 32 x 32 block, the rows below
//                  it by that inverse, the rest of the block by 4 x 4
//                  register tiles),
//                  writes L11 back and leaves the inverses of its 32 x 32
//                  diagonal blocks in the front's scratch slot;
//   k_panel_trsm   the rows below the block, L21 = A21 L11^{-T}, by blocked
//                  substitution with L11 and those inverses: 128-row items
//                  over a persistent grid of two CTAs per SM, 16 outputs
//                  per thread in registers.
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

// Scratch of warp_chol / warp_inv in shared memory (16-byte aligned): the
// factor transposed, LT[t * 36 + i] = L(i, t), then four columns of the
// factor, lane-major (cb[4 i + u] = L(i, jj + u)).
constexpr int kLT = 36;
constexpr int kCholScratch = 32 * kLT + 128;

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
  return ((size_t)2 * W * diag_stride<W>() + kCholScratch) * sizeof(T);
}
template <class T, int W>
constexpr size_t trsm_smem() {   // tile, off-diagonal blocks of L11, block inverses
  return ((size_t)W * xs_stride<T>() + (size_t)(W / 32) * (W / 32 - 1) / 2 * 1024 +
          (size_t)W * 32) * sizeof(T);
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

// Four consecutive values to 16-byte aligned shared memory.
__device__ __forceinline__ void st4(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ __forceinline__ void st4(double* p, double a, double b, double c, double d) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
  *reinterpret_cast<double2*>(p + 2) = make_double2(c, d);
}

// One element global -> shared without a register round trip (cp.async, so
// that a thread has dozens of loads in flight); zero-filled when !take.
__device__ __forceinline__ void cp_elem(float* dst, const float* src, bool take) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(take ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_elem(double* dst, const double* src, bool take) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(take ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One warp factors the jb x jb (jb <= 32) diagonal block at (j0, j0) of Ds
// (row-major, stride S) in place: lane i holds row i in registers.  Four
// columns at a time: their pivots and their mutual updates by shuffles, then
// the four columns of every lane go through shared memory once and the
// columns to the right take one rank-4 update (four values per load), so the
// warp makes one shared-memory round trip per four columns.  Leaves the factor
// transposed in Wk (LT[t * 36 + i] = L(i, t)).  Returns the first
// non-positive pivot column of the block, or -1.
template <class T, int JJ>
__device__ __forceinline__ void chol_cols4(T (&row)[32], int lane, int jb, T* cb, int& bad) {
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int j = JJ + u;
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
      for (int l = j + 1; l < JJ + 4; l++) {   // the rest of the four columns
        const T llj = __shfl_sync(0xffffffffu, row[j], l);
        if (lane >= l && l < jb) row[l] -= row[j] * llj;
      }
    }
  }
  if (JJ + 4 < 32) {
    st4(cb + 4 * lane, row[JJ], row[JJ + 1], row[JJ + 2], row[JJ + 3]);
    __syncwarp();
#pragma unroll
    for (int l = JJ + 4; l < 32; l++) {      // rank-4 update of the columns to the right
      T v[4];
      ld4(cb + 4 * l, v);
      if (lane >= l && l < jb) {
        T acc = row[l];
        acc = fma(-row[JJ], v[0], acc);
        acc = fma(-row[JJ + 1], v[1], acc);
        acc = fma(-row[JJ + 2], v[2], acc);
        row[l] = fma(-row[JJ + 3], v[3], acc);
      }
    }
    __syncwarp();                          // cb is rewritten by the next four columns
  }
}

template <class T, int S>
__device__ int warp_chol(T* Ds, int j0, int jb, T* Wk) {
  const int lane = threadIdx.x & 31;
  T* LT = Wk;
  T* cb = Wk + 32 * kLT;
  T row[32];
#pragma unroll
  for (int t = 0; t < 32; t++)
    row[t] = (lane < jb && t <= lane) ? Ds[(j0 + lane) * S + j0 + t] : T(0);
  int bad = -1;
  chol_cols4<T, 0>(row, lane, jb, cb, bad);
  chol_cols4<T, 4>(row, lane, jb, cb, bad);
  chol_cols4<T, 8>(row, lane, jb, cb, bad);
  chol_cols4<T, 12>(row, lane, jb, cb, bad);
  chol_cols4<T, 16>(row, lane, jb, cb, bad);
  chol_cols4<T, 20>(row, lane, jb, cb, bad);
  chol_cols4<T, 24>(row, lane, jb, cb, bad);
  chol_cols4<T, 28>(row, lane, jb, cb, bad);
#pragma unroll
  for (int t = 0; t < 32; t++) {
    if (lane < jb && t <= lane) Ds[(j0 + lane) * S + j0 + t] = row[t];
    LT[t * kLT + lane] = row[t];
  }
  __syncwarp();
  return bad;
}

// One warp: the inverse of the jb x jb factor left in Wk by warp_chol, to Li
// (row-major, stride LS; zero above the diagonal and outside jb).  Lane c
// holds column c and eliminates right-looking four rows at a time: the 4 x 4
// diagonal block, then a rank-4 update of the rows below it (four values per
// load of the transposed factor).
template <class T, int LS>
__device__ void warp_inv(const T* Wk, int jb, T* Li) {
  const int lane = threadIdx.x & 31;
  const T* LT = Wk;
  const T rd = lane < jb ? T(1) / LT[lane * kLT + lane] : T(1);
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) x[i] = i == lane ? T(1) : T(0);
#pragma unroll
  for (int tt = 0; tt < 32; tt += 4) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int t = tt + u;
      if (t < jb) {
        x[t] *= __shfl_sync(0xffffffffu, rd, t);
#pragma unroll
        for (int i = t + 1; i < tt + 4; i++)
          if (i < jb) x[i] -= LT[t * kLT + i] * x[t];
      }
    }
#pragma unroll
    for (int i4 = tt + 4; i4 < 32; i4 += 4) {
      T v0[4], v1[4], v2[4], v3[4];
      ld4(LT + (tt + 0) * kLT + i4, v0);
      ld4(LT + (tt + 1) * kLT + i4, v1);
      ld4(LT + (tt + 2) * kLT + i4, v2);
      ld4(LT + (tt + 3) * kLT + i4, v3);
#pragma unroll
      for (int w = 0; w < 4; w++) {
        if (i4 + w < jb) {
          T acc = x[i4 + w];
          acc = fma(-v0[w], x[tt], acc);
          acc = fma(-v1[w], x[tt + 1], acc);
          acc = fma(-v2[w], x[tt + 2], acc);
          x[i4 + w] = fma(-v3[w], x[tt + 3], acc);
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 32; i++) Li[i * LS + lane] = (i < jb && lane < jb && i >= lane) ? x[i] : T(0);
}

// 4 x 4 tiles of the lower triangle of the trailing block rows/columns
// [c1, kb): A(r, c) -= sum_t L(r, c0 + t) L(c, c0 + t), c <= r, for the tiles
// tI = first, first + step, ... below last (lower-triangle tile index).
template <class T, int S>
__device__ __forceinline__ void trail_tiles(T* As, int c0, int c1, int kb, int first, int last,
                                            int step) {
  for (int tI = first; tI < last; tI += step) {
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
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (ra + i < kb && ca + j <= ra + i) As[(ra + i) * S + ca + j] -= acc[i][j];
  }
}

// The kb x kb diagonal block of every front's panel, a CTA per front,
// right-looking over 32-column blocks: warp 0 factors block b and inverts it
// (registers, shared-memory broadcasts), then all warps form the rows below it
// as products with that inverse (a warp per eight rows, independent
// accumulators) and update the rest of the block (4 x 4 register tiles).  The
// phases do not overlap: the tile updates' shared-memory traffic would stretch
// the warp's latency-bound chain (measured slower).  Writes L11 into the front
// (lower triangle) and the inverses of its 32 x 32 diagonal blocks into the
// front's slot, K-major: slot[b 1024 + t 32 + c] = Li_b(c, t), zero outside
// the block's jb x jb lower triangle.
template <class T, int W>
__global__ void __launch_bounds__(kPanThreads) k_diag_factor(const int* __restrict__ flist,
                                                             const FrontDev* __restrict__ fr,
                                                             T* __restrict__ F, int Ks,
                                                             T* __restrict__ slot, DevError* err) {
  constexpr int S = diag_stride<W>(), NW = kPanThreads / 32;
  constexpr int MQ = (W - 32) / NW;         // rows below a block per warp, at most
  extern __shared__ __align__(16) unsigned char diag_raw[];
  T* As = reinterpret_cast<T*>(diag_raw);   // the block, then L11 (row-major, stride S)
  T* Vs = As + W * S;                       // inverses of the diagonal blocks (row-major, S)
  T* Wk = Vs + W * S;                       // warp_chol / warp_inv scratch
  __shared__ int badcol;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const FrontDev d = fr[flist[blockIdx.x]];
  if (Ks >= d.n) return;
  T* A = F + d.off;
  const int64_t ld = d.ld;
  const int kb = min(W, d.n - Ks), nb = (kb + 31) / 32;
  for (int idx = tid; idx < W * W; idx += kPanThreads) {
    const int r = idx % W, c = idx / W;
    const bool take = r < kb && c <= r;
    cp_elem(As + r * S + c, take ? A + (Ks + r) + (int64_t)(Ks + c) * ld : A, take);
  }
  cp_commit();
  if (tid == 0) badcol = -1;
  cp_wait<0>();
  __syncthreads();
  for (int b = 0; b < nb; b++) {
    const int c0 = 32 * b, jb = min(32, kb - c0), c1 = c0 + jb;
    if (warp == 0) {
      const int bad = warp_chol<T, S>(As, c0, jb, Wk);
      warp_inv<T, S>(Wk, jb, Vs + c0 * S + c0);
      if (lane == 0 && bad >= 0 && badcol < 0) badcol = Ks + c0 + bad;
    }
    __syncthreads();
    if (c1 >= kb) break;                    // the last block: nothing below it
    // rows below block b (jb = 32): L(r, c0 + c) = sum_t A(r, c0 + t) Li_b(c, t)
    {
      T acc[MQ];
#pragma unroll
      for (int q = 0; q < MQ; q++) acc[q] = T(0);
#pragma unroll 4
      for (int t = 0; t < 32; t++) {
        const T l = Vs[(c0 + lane) * S + c0 + t];
#pragma unroll
        for (int q = 0; q < MQ; q++) {
          const int r = c1 + warp + NW * q;
          if (r < kb) acc[q] = fma(As[r * S + c0 + t], l, acc[q]);
        }
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < MQ; q++) {
        const int r = c1 + warp + NW * q;
        if (r < kb) As[r * S + c0 + lane] = acc[q];
      }
    }
    __syncthreads();
    const int m4 = (kb - c1 + 3) / 4;
    trail_tiles<T, S>(As, c0, c1, kb, tid, m4 * (m4 + 1) / 2, kPanThreads);
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
  T* Li = slot + (int64_t)blockIdx.x * W * W;
  for (int idx = tid; idx < W * 32; idx += kPanThreads) {
    const int bq = idx >> 10, t = (idx >> 5) & 31, c = idx & 31;
    Li[idx] = bq < nb ? Vs[(32 * bq + c) * S + 32 * bq + t] : T(0);
  }
}

// The rows below the diagonal block, L21 = A21 L11^{-T}, over a persistent
// grid of two CTAs per SM.  Items are 128-row blocks of every front's rows
// [Ks + kb, N), listed front by front; a CTA takes items blockIdx.x,
// + gridDim.x, ...  The tile is K-major (X[c][r], fetched with cp.async);
// the off-diagonal 32 x 32 blocks of L11 (K-major inside each block, read
// from the front) and the inverses of its diagonal blocks (from the slot) are
// fetched once per front the CTA visits - only what the substitution reads,
// so that two CTAs fit an SM and one computes while the other waits for its
// tile.  Blocked substitution, 32 columns at a time: Y_b = X_b - sum_{k<b}
// Z_k L_bk^T, then Z_b = Y_b Li_b^T, written over X_b.  Thread (tx, ty) owns
// rows 4 ty .. 4 ty + 3 and 64 + the same, and in block b the columns
// 32 b + tx and 32 b + tx + 16, in registers.
template <class T, int W>
__global__ void __launch_bounds__(kPanThreads, 2) k_panel_trsm(const int* __restrict__ flist,
                                                               int nf,
                                                               const FrontDev* __restrict__ fr,
                                                               T* __restrict__ F, int Ks,
                                                               const T* __restrict__ slot) {
  constexpr int XS = xs_stride<T>(), NB = W / 32;
  extern __shared__ __align__(16) unsigned char trsm_raw[];
  T* X = reinterpret_cast<T*>(trsm_raw);    // the tile, K-major
  T* Lp = X + W * XS;                        // block (b, k < b) of L11 at (b (b - 1) / 2 + k) 1024
  T* Lis = Lp + NB * (NB - 1) / 2 * 1024;    // inverses of its diagonal blocks, K-major
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
      for (int idx = tid; idx < NB * (NB - 1) / 2 * 1024; idx += kPanThreads) {
        const int blk = idx >> 10, tt = (idx >> 5) & 31, cc = idx & 31;
        int b = 1;
        while ((b + 1) * b / 2 <= blk) b++;  // block row b of packed block blk
        const int k = blk - b * (b - 1) / 2;
        const int c = 32 * b + cc, t = 32 * k + tt;
        const bool take = c < kb && t < kb;
        cp_elem(Lp + idx, take ? A + (Ks + c) + (int64_t)(Ks + t) * ld : A, take);
      }
      const T* Lt = slot + (int64_t)i * W * W;
      for (int idx = tid; idx < W * 32; idx += kPanThreads) cp_elem(Lis + idx, Lt + idx, true);
    }
    for (int idx = tid; idx < W * kTrsmRows; idx += kPanThreads) {
      const int r = idx % kTrsmRows, t = idx / kTrsmRows;
      const bool take = r < rows && t < kb;
      cp_elem(X + t * XS + r, take ? A + (r0 + r) + (int64_t)(Ks + t) * ld : A, take);
    }
    cp_commit();
    cp_wait<0>();
    __syncthreads();
    const int nbk = (kb + 31) / 32;
    for (int b = 0; b < nbk && b < NB; b++) {
      const int ca = 32 * b + tx, cb = ca + 16;
      T acc[8][2];
      {
        T xa[8], xb[8];                      // X_b, the thread's two columns
        ld4(X + ca * XS + 4 * ty, xa);
        ld4(X + ca * XS + 64 + 4 * ty, xa + 4);
        ld4(X + cb * XS + 4 * ty, xb);
        ld4(X + cb * XS + 64 + 4 * ty, xb + 4);
#pragma unroll
        for (int r = 0; r < 8; r++) {
          acc[r][0] = xa[r];
          acc[r][1] = xb[r];
        }
      }
      for (int k = 0; k < b; k++) {          // - Z_k L_bk^T over the solved blocks
        const T* Lb = Lp + (b * (b - 1) / 2 + k) * 1024;
#pragma unroll 4
        for (int tt = 0; tt < 32; tt++) {
          T z[8];
          ld4(X + (32 * k + tt) * XS + 4 * ty, z);
          ld4(X + (32 * k + tt) * XS + 64 + 4 * ty, z + 4);
          const T la = Lb[tt * 32 + tx], lb = Lb[tt * 32 + tx + 16];
#pragma unroll
          for (int r = 0; r < 8; r++) {
            acc[r][0] = fma(-z[r], la, acc[r][0]);
            acc[r][1] = fma(-z[r], lb, acc[r][1]);
          }
        }
      }
      // Y_b in place (only this thread reads these entries before the barrier)
#pragma unroll
      for (int r = 0; r < 8; r++) {
        X[ca * XS + 64 * (r >> 2) + 4 * ty + (r & 3)] = acc[r][0];
        X[cb * XS + 64 * (r >> 2) + 4 * ty + (r & 3)] = acc[r][1];
      }
      __syncthreads();
      // Z_b = Y_b Li_b^T
      T out[8][2];
#pragma unroll
      for (int r = 0; r < 8; r++) out[r][0] = out[r][1] = T(0);
      const T* Li = Lis + b * 1024;
#pragma unroll 4
      for (int t = 0; t < 32; t++) {
        T y[8];
        ld4(X + (32 * b + t) * XS + 4 * ty, y);
        ld4(X + (32 * b + t) * XS + 64 + 4 * ty, y + 4);
        const T la = Li[t * 32 + tx], lb = Li[t * 32 + tx + 16];
#pragma unroll
        for (int r = 0; r < 8; r++) {
          out[r][0] = fma(y[r], la, out[r][0]);
          out[r][1] = fma(y[r], lb, out[r][1]);
        }
      }
      __syncthreads();                       // every read of Y_b is done
#pragma unroll
      for (int r = 0; r < 8; r++) {
        X[ca * XS + 64 * (r >> 2) + 4 * ty + (r & 3)] = out[r][0];
        X[cb * XS + 64 * (r >> 2) + 4 * ty + (r & 3)] = out[r][1];
      }
      __syncthreads();
    }
    for (int idx = tid; idx < kb * kTrsmRows; idx += kPanThreads) {
      const int r = idx % kTrsmRows, c = idx / kTrsmRows;
      if (r < rows) A[(r0 + r) + (int64_t)(Ks + c) * ld] = X[c * XS + r];
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
