// Tensor-core trailing update of the mixed-precision factorization (sm_100a).
//
// After a panel of w pivot columns [K, k1) of a front has been factored
// (k1 = min(K + w, n)), the rest of the front is updated by
//     C(k1:N, k1:cmax) -= P P(k1:cmax)^T,   P = L(k1:N, K:k1)
// (lower triangle only), the right-looking Cholesky step that the reference's
// dense LU performs inside Factor() (src/DE/mf2d.cpp:792-901, via
// LinAlg::Dense::LU).  cmax = N for the trailing update after an outer panel
// (w = 512); inside an outer panel [K0, K0 + 512) the update after each
// 128-column sub-panel is limited to the outer panel's remaining columns,
// cmax = min(K0 + 512, n).  For the large fronts of the top tree levels this
// is nearly all of the work.
//
// Two kernels per panel:
//   * k_tc_pack writes the panel once, split into TF32 "hi" and "lo" parts
//     (x = hi + lo, both exactly representable), as 8 KB images of 128 rows x
//     16 columns in the K-major 64-byte-swizzled layout the tensor core reads:
//     one CTA per (128-row block, 16-column chunk) reads its block coalesced
//     from the column-major front and splits it in shared memory; per chunk
//     the hi images of all row blocks are contiguous, then the lo images;
//   * k_trail_tc, a persistent warp-specialised pipeline over 128 x 256 tiles
//     of C (block row I of 128 rows, block column J of 256 columns, lower
//     triangle only):
//       - one producer thread brings each chunk's images (the tile's row
//         block, unless it lies inside the column block, and the two row
//         blocks of the column block) into a ring of four shared-memory
//         stages with bulk asynchronous copies (cp.async.bulk, completion
//         counted in bytes on an mbarrier);
//       - one MMA warp issues tcgen05.mma (kind::tf32, M = 128, N = 256,
//         K = 8) from an elected lane into one of two tensor-memory
//         accumulators (256 columns each, all of tensor memory):
//             SPLIT = 3:  acc += hi_a hi_b^T + hi_a lo_b^T + lo_a hi_b^T
//             SPLIT = 1:  acc += hi_a hi_b^T
//             SPLIT = 2:  acc += a b^T in BF16 (kind::f16, K = 16; the pack
//                         writes BF16 images of 32 columns, the same 8 KB size)
//         and hands stages back to the producer with tcgen05.commit;
//       - eight epilogue warps (two per accumulator lane quarter, 128 columns
//         each, 32 at a time) read the accumulator with tcgen05.ld and
//         subtract it from C in place; the first 32 values of C are loaded
//         before the accumulator is ready.
// A 256-column tile reads 25% fewer operand bytes per product than a 128 x 128
// one, and 16-column stages keep three stages in flight.  MN-major TF32
// operands would let the tensor core read the column-major front directly,
// but they read back as zeros on sm_100a, hence the pack.  The three-term form
// keeps products to about 2^-21 relative error, close to FP32.
//
// Every mbarrier wait is bounded (kSpinLimit polls, or the limit the host put
// in the error word); on expiry (or once another warp gave up) the kernel
// records error code 2 in the error word, skips the remaining work, waits for
// its own copies and products in flight, releases its tensor memory and
// returns.
#include <cuda_bf16.h>

#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int TM = 128;                    // C tile rows = accumulator lanes = image rows
constexpr int TN = 256;                    // C tile columns = accumulator columns
constexpr int TK = 16;                     // TF32: panel columns per chunk (64-byte image rows)
constexpr int TK16 = 32;                   // BF16: panel columns per chunk (64-byte image rows)
constexpr int NSTAGE = 4;                  // shared-memory stages
constexpr int NACC = 2;                    // tensor-memory accumulators
constexpr int MMA_WARP = 1;                // warp 0 produces, warp 1 issues the MMAs
constexpr int EPI_WARP0 = 2;               // warps 2..9 run the epilogue
constexpr int NEPI = 8;
constexpr int TCT = (EPI_WARP0 + NEPI) * 32;   // 320 threads
constexpr int IMG = TM * TK * 4;           // one image of 128 rows x 16 columns, 8 KB
constexpr int STAGE_BYTES = 6 * IMG;       // a_hi, a_lo, b_hi (2 blocks), b_lo (2 blocks)
constexpr int kTcSmem = NSTAGE * STAGE_BYTES + 1024;   // + alignment slack
constexpr int kMaxTcFronts = 1024;
constexpr int kTcOuter = 512;              // outer panel width (the cooperative kernel's)
constexpr uint32_t kSpinLimit = 1u << 24;

// Image layout (K-major, 64-byte swizzle): element (m, k) of a 128 x 16 image
// sits in 64-byte row m, 16-byte chunk (k / 4) ^ ((m / 2) % 4), word k % 4;
// 8-row groups are 512 bytes apart.
__host__ __device__ constexpr int img_off(int m, int k) {
  return m * 64 + ((((k >> 2) ^ ((m >> 1) & 3))) << 4) + (k & 3) * 4;
}

// Instruction descriptors: D = F32, both operands K-major, M = 128, N = 256;
// A = B = TF32 (kind::tf32) or A = B = BF16 (kind::f16; never mixed types).
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                                ((uint32_t)(TM >> 4) << 24);

// Panel columns per chunk of each mode: SPLIT = 3 three-term TF32, 1 plain
// TF32 (16 columns), 2 plain BF16 (one product, 32 columns).
__host__ __device__ constexpr int chunk_cols(int split) { return split == 2 ? TK16 : TK; }

// Panel geometry of a front for the panel [K, K + w): k1, 128-row blocks
// below k1, 16-column chunks in [K, k1), the column bound cmax (cend < 0: N,
// else min(cend, n)) and the 256-column blocks of C left of it; nb = 0 when
// the front has no update.  Tiles: block rows I < nb, block columns
// J <= I / 2, J < nj.
struct PanelGeo {
  int k1, nb, nch, cmax, nj;
};
__host__ __device__ inline PanelGeo panel_geo(int n, int N, int K, int w, int cend, int tk = TK) {
  PanelGeo g{0, 0, 0, 0, 0};
  if (K >= n) return g;
  g.k1 = n < K + w ? n : K + w;
  if (N <= g.k1) return g;
  g.cmax = cend < 0 ? N : (cend < n ? cend : n);
  if (g.cmax <= g.k1) return g;
  g.nb = (N - g.k1 + TM - 1) / TM;
  g.nch = (g.k1 - K + tk - 1) / tk;
  g.nj = (g.cmax - g.k1 + TN - 1) / TN;   // <= (nb + 1) / 2 since cmax <= N
  return g;
}

// Tiles of a front: row I has min(I / 2 + 1, nj) of them.  Rows 0 .. 2 nj - 1
// come in pairs (2p, 2p + 1) of p + 1 tiles each; the rows below have nj.
__host__ __device__ inline int geo_tiles(const PanelGeo& g) {
  if (g.nb <= 2 * g.nj) {
    const int p = g.nb / 2;
    return g.nb % 2 == 0 ? p * (p + 1) : (p + 1) * (p + 1);
  }
  return g.nj * (g.nj + 1) + (g.nb - 2 * g.nj) * g.nj;
}

// Tile order.  The tiles of a front ({(I, J): I < nb, J < nj, 2 J <= I})
// come in groups of kTileGroup block rows; inside group [a, b) block column J
// runs outer and the rows max(a, 2 J) .. b - 1 inner.  The CTAs working at
// the same time then share one or two column blocks of B and revisit the
// group's rows of A, whose packed images (16 MB per 32 rows at K = 512) stay
// in L2; in plain row order they sweep every column block of the panel, which
// for the largest fronts (a 196 MB panel at 127^3) does not fit in L2.
constexpr int kTileGroup = 32;

// Columns of group [a, b) holding all its rows (2 J <= a) and holding some.
__host__ __device__ inline void group_cols(int a, int b, int nj, int& jf, int& je) {
  jf = a / 2 + 1 < nj ? a / 2 + 1 : nj;
  je = (b - 1) / 2 + 1 < nj ? (b - 1) / 2 + 1 : nj;
}
// Tiles in the first k partial columns (column jf + i holds b - 2 (jf + i)).
__host__ __device__ inline int partial_tiles(int b, int jf, int k) {
  return k * (b - 2 * jf) - k * (k - 1);
}

__host__ __device__ inline void tile_ij(int t, int nb, int nj, int& I, int& J) {
  int a = 0, b = 0, jf = 0, je = 0;
  for (a = 0; a < nb; a += kTileGroup) {
    b = a + kTileGroup < nb ? a + kTileGroup : nb;
    group_cols(a, b, nj, jf, je);
    const int T = jf * (b - a) + partial_tiles(b, jf, je - jf);
    if (t < T) break;
    t -= T;
  }
  const int h = b - a;
  if (t < jf * h) {
    J = t / h;
    I = a + t % h;
    return;
  }
  t -= jf * h;
  const double c1 = (double)(b - 2 * jf) + 1.0;   // partial_tiles(k) = k (c1 - k)
  int k = (int)((c1 - sqrt(c1 * c1 - 4.0 * (double)t)) * 0.5);
  if (k < 0) k = 0;
  while (k > 0 && partial_tiles(b, jf, k) > t) k--;
  while (partial_tiles(b, jf, k + 1) <= t) k++;
  J = jf + k;
  I = 2 * J + (t - partial_tiles(b, jf, k));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major operand image with 64-byte
// swizzle: rows of 64 bytes, 8-row groups 512 bytes apart.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

// Bulk asynchronous copy global -> this CTA's shared memory; completion is
// counted in bytes on the mbarrier (addresses 16-byte aligned, size a
// multiple of 16).
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Arrive on the mbarrier and add `bytes` to the transaction count its
// current phase waits for.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Wait for completion of the mbarrier phase with the given parity.  Bounded:
// returns false after `limit` polls or as soon as *abort is set.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                                          uint32_t limit) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255 && *abort) return false;
  }
  *abort = 1;
  return false;
}

// Warp-uniform wait: lane 0 polls, the outcome is broadcast to the warp so that
// the warp's collective tcgen05 instructions stay converged.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort,
                                               uint32_t limit) {
  bool ok = true;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort, limit);
  return __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdescBf16), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive accumulator columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Tile t of the launch: front slot i, block row I, block column J.
struct TileInfo {
  float* A;
  int64_t ld;
  int N, k1, cmax, r0, c0, nch, nb, slot, I, J;
};

__device__ __forceinline__ TileInfo tile_info(const int* pre, int nf, const int* flist,
                                              const FrontDev* fr, float* F, int K, int w, int cend,
                                              int tile, int tk) {
  int lo = 0, hi = nf - 1;   // largest i with pre[i] <= tile
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= tile) lo = mid;
    else hi = mid - 1;
  }
  const FrontDev d = fr[flist[lo]];
  const PanelGeo g = panel_geo(d.n, d.N, K, w, cend, tk);
  TileInfo t;
  t.A = F + d.off;
  t.ld = d.ld;
  t.N = d.N;
  t.k1 = g.k1;
  t.cmax = g.cmax;
  t.nch = g.nch;
  t.nb = g.nb;
  t.slot = lo;
  tile_ij(tile - pre[lo], g.nb, g.nj, t.I, t.J);
  t.r0 = t.k1 + t.I * TM;
  t.c0 = t.k1 + t.J * TN;
  return t;
}

// Pack: CTA (x, i) = chunk c, row block b (x = c * nb + b) of front slot i:
// rows k1 + 128 b + t (thread t), columns K + 16 c .. +15; zeros outside the
// front and beyond k1.  Front slot i owns bytes [i * cap * 2 * IMG, +cap * 2 *
// IMG) of pack; inside, the hi image of (c, b) is image (2 c) * nb + b and the
// lo image (2 c + 1) * nb + b.
template <int SPLIT>
__global__ void __launch_bounds__(128) k_tc_pack(const int* __restrict__ flist,
                                                 const FrontDev* __restrict__ fr,
                                                 const float* __restrict__ F, int K, int w,
                                                 int cap, unsigned char* __restrict__ pack) {
  __shared__ __align__(1024) unsigned char img[2 * IMG];
  const FrontDev d = fr[flist[blockIdx.y]];
  constexpr int tk = chunk_cols(SPLIT);
  const PanelGeo g = panel_geo(d.n, d.N, K, w, -1, tk);
  const int x = blockIdx.x;
  if (x >= g.nb * g.nch) return;
  const int c = x / g.nb, b = x - c * g.nb, t = threadIdx.x;
  const int row = g.k1 + b * TM + t, kc = K + c * tk;
  const bool row_ok = row < d.N;
  const float* src = F + d.off + (row_ok ? row : 0) + (int64_t)kc * d.ld;
  const int kend = g.k1 - kc;   // columns of this chunk inside the panel
  if (SPLIT == 2) {
    // BF16 (round to nearest even): 32 columns, 16-byte chunks of 8 values,
    // the 64-byte swizzle of the TF32 images on 16-byte units
#pragma unroll
    for (int q = 0; q < TK16 / 8; q++) {
      uint32_t pk[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int k0 = 8 * q + 2 * j;
        const float v0 = (row_ok && k0 < kend) ? __ldg(src + (int64_t)k0 * d.ld) : 0.0f;
        const float v1 = (row_ok && k0 + 1 < kend) ? __ldg(src + (int64_t)(k0 + 1) * d.ld) : 0.0f;
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(v0, v1);   // .x = v0 at the lower address
        pk[j] = *reinterpret_cast<const uint32_t*>(&h2);
      }
      *reinterpret_cast<uint4*>(img + t * 64 + ((q ^ ((t >> 1) & 3)) << 4)) =
          make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  } else {
#pragma unroll
  for (int q = 0; q < TK / 4; q++) {
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * q + j;
      v[j] = (row_ok && k < kend) ? __ldg(src + (int64_t)k * d.ld) : 0.0f;
    }
    float4 h, l;
    h.x = tf32_round(v[0]);
    h.y = tf32_round(v[1]);
    h.z = tf32_round(v[2]);
    h.w = tf32_round(v[3]);
    *reinterpret_cast<float4*>(img + img_off(t, 4 * q)) = h;
    if (SPLIT == 3) {
      l.x = tf32_round(v[0] - h.x);
      l.y = tf32_round(v[1] - h.y);
      l.z = tf32_round(v[2] - h.z);
      l.w = tf32_round(v[3] - h.w);
      *reinterpret_cast<float4*>(img + IMG + img_off(t, 4 * q)) = l;
    }
  }
  }
  __syncthreads();
  unsigned char* base = pack + (int64_t)blockIdx.y * cap * 2 * IMG;
  float4* dh = reinterpret_cast<float4*>(base + ((int64_t)(2 * c) * g.nb + b) * IMG);
  float4* dl = reinterpret_cast<float4*>(base + ((int64_t)(2 * c + 1) * g.nb + b) * IMG);
  const float4* s4 = reinterpret_cast<const float4*>(img);
#pragma unroll
  for (int e = t; e < IMG / 16; e += 128) {
    dh[e] = s4[e];
    if (SPLIT == 3) dl[e] = s4[IMG / 16 + e];
  }
}

template <int SPLIT>
__global__ void __launch_bounds__(TCT, 1) k_trail_tc(const int* __restrict__ flist, int nf,
                                                     const FrontDev* __restrict__ fr,
                                                     float* __restrict__ F, int K, int w, int cend,
                                                     int cap, const unsigned char* __restrict__ pack,
                                                     DevError* err) {
  extern __shared__ unsigned char tc_raw[];
  __shared__ uint64_t full[NSTAGE], empty[NSTAGE], acc_full[NACC], acc_empty[NACC], drain;
  __shared__ uint32_t tmem_base;
  __shared__ int pre[kMaxTcFronts + 1];
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // pipeline waits give up after this many polls (host-settable); the waits
  // that drain work already issued before the CTA exits keep kSpinLimit
  const uint32_t lim = wait_limit(err, kSpinLimit);
  unsigned char* sm =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~(uintptr_t)1023);

  // tiles per front (in parallel), then their prefix (thread 0, shared memory)
  for (int i = tid; i < nf; i += TCT) {
    const FrontDev d = fr[flist[i]];
    pre[i + 1] = geo_tiles(panel_geo(d.n, d.N, K, w, cend));
  }
  __syncthreads();
  if (tid == 0) {
    pre[0] = 0;
    for (int i = 0; i < nf; i++) pre[i + 1] += pre[i];
    for (int s = 0; s < NSTAGE; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NACC; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], NEPI * 32);
    }
    mbar_init(&drain, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(NACC * TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  const int total = pre[nf];

  if (warp == 0) {
    // ---- producer: one thread fills the stages; stage layout: a_hi, a_lo,
    // b_hi (row blocks 2J, 2J + 1), b_lo (same) ----
    if (lane == 0) {
      const uint32_t sm0 = smem_u32(sm);
      uint32_t g = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < total && !abort_flag; tile += gridDim.x) {
        const TileInfo ti = tile_info(pre, nf, flist, fr, F, K, w, cend, tile, chunk_cols(SPLIT));
        const unsigned char* base = pack + (int64_t)ti.slot * cap * 2 * IMG;
        const int bb = 2 * ti.J, nbb = min(2, ti.nb - bb);   // row blocks of the column block
        const bool a_in_b = ti.I - bb < nbb;                   // row block I is one of them
        const uint32_t bbytes = (uint32_t)nbb * IMG, abytes = a_in_b ? 0u : (uint32_t)IMG;
        const uint32_t tx = (SPLIT == 3 ? 2 : 1) * (abytes + bbytes);
        for (int c = 0; c < ti.nch; c++, g++) {
          const int s = g % NSTAGE;
          const uint32_t u = g / NSTAGE;
          if (u >= 1 && !mbar_wait(&empty[s], (u - 1) & 1, &abort_flag, lim)) {
            ok = false;
            break;
          }
          const uint32_t st = sm0 + s * STAGE_BYTES;
          const unsigned char* hi = base + (int64_t)(2 * c) * ti.nb * IMG;
          const unsigned char* lo = base + (int64_t)(2 * c + 1) * ti.nb * IMG;
          mbar_expect_tx(&full[s], tx);
          bulk_copy(st + 2 * IMG, hi + (int64_t)bb * IMG, bbytes, &full[s]);
          if (SPLIT == 3) bulk_copy(st + 4 * IMG, lo + (int64_t)bb * IMG, bbytes, &full[s]);
          if (!a_in_b) {
            bulk_copy(st, hi + (int64_t)ti.I * IMG, IMG, &full[s]);
            if (SPLIT == 3) bulk_copy(st + IMG, lo + (int64_t)ti.I * IMG, IMG, &full[s]);
          }
        }
      }
      // the copies still in flight land before the CTA may exit
      volatile int never = 0;
      for (uint32_t q = g > NSTAGE ? g - NSTAGE : 0; q < g; q++)
        mbar_wait(&full[q % NSTAGE], (q / NSTAGE) & 1, &never, kSpinLimit);
    }
  } else if (warp == MMA_WARP) {
    // ---- MMA issue ----
    uint32_t g = 0, tl = 0;
    for (int tile = blockIdx.x; tile < total && !__shfl_sync(0xffffffffu, abort_flag, 0);
         tile += gridDim.x, tl++) {
      const TileInfo ti = tile_info(pre, nf, flist, fr, F, K, w, cend, tile, chunk_cols(SPLIT));
      const int b = tl % NACC;
      const uint32_t v = tl / NACC;
      if (v >= 1 && !mbar_wait_warp(&acc_empty[b], (v - 1) & 1, &abort_flag, lim)) break;
      tc_fence_after();
      const uint32_t dacc = tmem + b * TN;
      const int bb = 2 * ti.J, nbb = min(2, ti.nb - bb);
      const int ia = ti.I - bb;   // row block I inside the column block when 0 <= ia < nbb
      bool ok = true;
      for (int c = 0; c < ti.nch; c++, g++) {
        const int s = g % NSTAGE;
        if (!mbar_wait_warp(&full[s], (g / NSTAGE) & 1, &abort_flag, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t st = smem_u32(sm + s * STAGE_BYTES);
          const uint32_t b_hi = st + 2 * IMG, b_lo = st + 4 * IMG;
          const bool in = ia >= 0 && ia < nbb;
          const uint32_t a_hi = in ? b_hi + ia * IMG : st, a_lo = in ? b_lo + ia * IMG : st + IMG;
#pragma unroll
          for (int kk = 0; kk < 2; kk++) {
            // K = 8 TF32 or K = 16 BF16 values: 32 bytes along the swizzled row
            const uint32_t ko = kk * 32;
            if (SPLIT == 2) {
              mma_bf16(dacc, sw64_desc(a_hi + ko), sw64_desc(b_hi + ko), (c | kk) != 0);
              continue;
            }
            mma_tf32(dacc, sw64_desc(a_hi + ko), sw64_desc(b_hi + ko), (c | kk) != 0);
            if (SPLIT == 3) {
              mma_tf32(dacc, sw64_desc(a_hi + ko), sw64_desc(b_lo + ko), 1u);
              mma_tf32(dacc, sw64_desc(a_lo + ko), sw64_desc(b_hi + ko), 1u);
            }
          }
          mma_commit(&empty[s]);
        }
        __syncwarp();
      }
      if (!ok) break;
      if (lane == 0) mma_commit(&acc_full[b]);
      __syncwarp();
    }
    // after an abort, products already issued may still be running: a commit
    // tracks all of them, and tensor memory is released only once it fired
    if (abort_flag && g > 0) {
      if (lane == 0) mma_commit(&drain);
      __syncwarp();
      volatile int never = 0;
      mbar_wait_warp(&drain, 0, &never, kSpinLimit);
    }
  } else {
    // ---- epilogue: C(tile) -= acc; warp w reads accumulator lanes
    // 32 (w % 4) .. +31 (the lane quarter it may access), columns 128 h .. +127,
    // 32 at a time ----
    const int quarter = warp & 3, half = (warp - EPI_WARP0) >> 2;
    uint32_t tl = 0;
    for (int tile = blockIdx.x; tile < total && !__shfl_sync(0xffffffffu, abort_flag, 0);
         tile += gridDim.x, tl++) {
      const TileInfo ti = tile_info(pre, nf, flist, fr, F, K, w, cend, tile, chunk_cols(SPLIT));
      const int b = tl % NACC;
      const int row = ti.r0 + quarter * 32 + lane, cb = ti.c0 + half * (TN / 2);
      const bool live = row < ti.N;
      float* p = ti.A + row + (int64_t)cb * ti.ld;
      // entry j of the row is live when cb + j <= min(row, cmax - 1); the first
      // 32 values are loaded while the tile's products are still being
      // accumulated, each later 32 once the previous ones are stored
      const int jmax = live ? min(row, ti.cmax - 1) - cb : -1;
      const uint32_t src = tmem + b * TN + half * (TN / 2) + ((uint32_t)(quarter * 32) << 16);
      bool ok = true;
#pragma unroll 1
      for (int h2 = 0; h2 < TN / 64; h2++) {
        float cv[32];
        const float* q = p + (int64_t)(32 * h2) * ti.ld;
#pragma unroll
        for (int j = 0; j < 32; j++, q += ti.ld) cv[j] = 32 * h2 + j <= jmax ? *q : 0.0f;
        if (h2 == 0) {
          if (!mbar_wait_warp(&acc_full[b], (tl / NACC) & 1, &abort_flag, lim)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        float* wp = p + (int64_t)(32 * h2) * ti.ld;
#pragma unroll
        for (int qb = 0; qb < 2; qb++) {
          uint32_t v[16];
          tmem_ld16(src + 32 * h2 + 16 * qb, v);
#pragma unroll
          for (int j = 0; j < 16; j++, wp += ti.ld)
            if (32 * h2 + 16 * qb + j <= jmax) *wp = cv[16 * qb + j] - __uint_as_float(v[j]);
        }
      }
      if (!ok) break;
      tc_fence_before();
      mbar_arrive(&acc_empty[b]);
    }
  }
  if (abort_flag && tid == 0 && err) atomicCAS(&err->code, 0, 2);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == MMA_WARP)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(NACC * TN));
}

}  // namespace

int tc_outer() { return kTcOuter; }
int tc_max_fronts() { return kMaxTcFronts; }

int64_t tc_tiles(const std::vector<int>& n, const std::vector<int>& N, int K, int w, int cend) {
  int64_t t = 0;
  for (size_t i = 0; i < n.size(); i++) t += geo_tiles(panel_geo(n[i], N[i], K, w, cend));
  return t;
}

int tc_pack_cap(const std::vector<int>& n, const std::vector<int>& N, int K, int w) {
  int cap = 0;
  for (size_t i = 0; i < n.size(); i++) {
    const PanelGeo g = panel_geo(n[i], N[i], K, w, -1);
    cap = std::max(cap, g.nb * g.nch);
  }
  return cap;
}

size_t tc_pack_bytes(int nf, int cap) { return (size_t)nf * (size_t)cap * 2 * IMG; }

namespace {
int tc_setup() {   // thread-safe one-time set-up (static local initialisation)
  static const int sms = []() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_trail_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    cudaFuncSetAttribute(k_trail_tc<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    cudaFuncSetAttribute(k_trail_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    return n;
  }();
  return sms;
}
}  // namespace

cudaError_t launch_tc_pack(const int* flist, int nf, int cap, const FrontDev* fr, const float* F,
                           int K, int w, int split, void* pack, cudaStream_t st) {
  if (nf <= 0 || cap <= 0) return cudaSuccess;
  if (nf > 65535 || split < 1 || split > 3 || w <= 0 || w % chunk_cols(split) || w > kTcOuter)
    return cudaErrorInvalidValue;
  const dim3 grid((unsigned)cap, (unsigned)nf);
  if (split == 3)
    k_tc_pack<3><<<grid, 128, 0, st>>>(flist, fr, F, K, w, cap, (unsigned char*)pack);
  else if (split == 2)
    k_tc_pack<2><<<grid, 128, 0, st>>>(flist, fr, F, K, w, cap, (unsigned char*)pack);
  else
    k_tc_pack<1><<<grid, 128, 0, st>>>(flist, fr, F, K, w, cap, (unsigned char*)pack);
  g_launches++;
  return cudaGetLastError();
}

cudaError_t launch_trail_tc(const int* flist, int nf, int64_t ntiles, const FrontDev* fr, float* F,
                            int K, int w, int cend, int split, int cap, const void* pack,
                            DevError* err, cudaStream_t st) {
  if (nf <= 0 || ntiles <= 0) return cudaSuccess;
  if (nf > kMaxTcFronts || split < 1 || split > 3 || !pack || w <= 0 ||
      w % chunk_cols(split) || w > kTcOuter)
    return cudaErrorInvalidValue;
  const int grid = (int)std::min<int64_t>(ntiles, tc_setup());
  if (split == 3)
    k_trail_tc<3><<<grid, TCT, kTcSmem, st>>>(flist, nf, fr, F, K, w, cend, cap,
                                              (const unsigned char*)pack, err);
  else if (split == 2)
    k_trail_tc<2><<<grid, TCT, kTcSmem, st>>>(flist, nf, fr, F, K, w, cend, cap,
                                              (const unsigned char*)pack, err);
  else
    k_trail_tc<1><<<grid, TCT, kTcSmem, st>>>(flist, nf, fr, F, K, w, cend, cap,
                                              (const unsigned char*)pack, err);
  g_launches++;
  return cudaGetLastError();
}

}  // namespace mfgpu
