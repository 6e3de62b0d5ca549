// Tensor-core trailing update of the mixed-precision factorization (sm_100a).
//
// After an outer panel of 512 pivot columns [K, k1) of a front has been
// factored (k1 = min(K + 512, n)), the rest of the front is updated by
//     C(k1:N, k1:N) -= P P^T,   P = L(k1:N, K:k1)
// (lower triangle only), the right-looking Cholesky step that the reference's
// dense LU performs inside Factor() (src/DE/mf2d.cpp:792-901, via
// LinAlg::Dense::LU).  For the large fronts of the top tree levels this is
// nearly all of the work.
//
// Each CTA is a persistent, warp-specialised pipeline over 128 x 128 tiles of
// C (lower triangle only):
//   * three loader warpgroups take the 32-column panel chunks in turn: each
//     reads 128 rows x 32 columns of the panel for the tile's rows (and, off
//     the diagonal, for its columns), splits them into TF32 "hi" and "lo"
//     parts (x = hi + lo, both exactly representable after rounding) and
//     writes them to its own shared-memory stage in the K-major 128-byte
//     swizzled layout the tensor core reads;
//   * one MMA warp issues tcgen05.mma (kind::tf32, M = N = 128, K = 8) from an
//     elected lane into one of two tensor-memory accumulators:
//         SPLIT = 3:  acc += hi_a hi_b^T + hi_a lo_b^T + lo_a hi_b^T
//         SPLIT = 1:  acc += hi_a hi_b^T
//     and hands stages back to the loaders with tcgen05.commit;
//   * four epilogue warps read the other accumulator with tcgen05.ld and
//     subtract it from C in place, with the next columns' loads of C in
//     flight while the current ones are stored.
// The three-term form keeps products to about 2^-21 relative error, close to
// FP32.
//
// Every mbarrier wait is bounded; on expiry (or once another warp gave up) the
// kernel records error code 2 in the error word, skips the remaining work,
// releases its tensor memory and returns.
#include <atomic>
#include <cstdint>

#include "device.cuh"

namespace mfgpu {

extern std::atomic<long long> g_launches;

namespace {

constexpr int TM = 128;                    // C tile rows = accumulator lanes
constexpr int TN = 128;                    // C tile columns = accumulator columns
constexpr int TK = 32;                     // panel columns per stage (128-byte rows)
constexpr int NLOAD = 3;                   // loader warpgroups = shared-memory stages
constexpr int NSTAGE = NLOAD;
constexpr int NACC = 2;                    // tensor-memory accumulators
constexpr int MMA_WARP = NLOAD * 4;        // warp 12 issues the MMAs
constexpr int EPI_WARP0 = MMA_WARP + 1;    // warps 13..16 run the epilogue
constexpr int TCT = (EPI_WARP0 + 4) * 32;  // 544 threads
constexpr int IMG = TM * TK * 4;           // one operand image, 16 KB
constexpr int STAGE_BYTES = 4 * IMG;       // a_hi, a_lo, b_hi, b_lo
constexpr int kTcSmem = NSTAGE * STAGE_BYTES + 1024;   // + alignment slack
constexpr int kMaxTcFronts = 1024;
constexpr int kTcOuter = 512;              // outer panel width (the cooperative kernel's)
constexpr uint32_t kSpinLimit = 1u << 24;

// Instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major operand image with 128-byte
// swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Wait for completion of the mbarrier phase with the given parity.  Bounded:
// returns false after kSpinLimit polls or as soon as *abort is set.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kSpinLimit; it++) {
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
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort) {
  bool ok = true;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort);
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

__device__ __forceinline__ void tri_ij(int t, int& I, int& J) {
  I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while (I * (I + 1) / 2 > t) I--;
  while ((I + 1) * (I + 2) / 2 <= t) I++;
  J = t - I * (I + 1) / 2;
}

// Tile t of the launch: front slot lo, block row I >= block column J.
struct TileInfo {
  float* A;
  int64_t ld;
  int N, k1, r0, c0, nch;
  bool diag;
};

__device__ __forceinline__ TileInfo tile_info(const int* pre, int nf, const int* flist,
                                              const FrontDev* fr, float* F, int K, int tile) {
  int lo = 0, hi = nf - 1;   // largest i with pre[i] <= tile
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= tile) lo = mid;
    else hi = mid - 1;
  }
  const FrontDev d = fr[flist[lo]];
  TileInfo t;
  t.A = F + d.off;
  t.ld = d.ld;
  t.N = d.N;
  t.k1 = min(K + kTcOuter, d.n);
  int I, J;
  tri_ij(tile - pre[lo], I, J);
  t.r0 = t.k1 + I * TM;
  t.c0 = t.k1 + J * TN;
  t.diag = (I == J);
  t.nch = (t.k1 - K + TK - 1) / TK;
  return t;
}

// 16 values of C for one row: columns cb .. cb+15 inside the lower triangle.
__device__ __forceinline__ void c_load(const float* p, int64_t ld, int row, int cb, int N,
                                       float (&c)[16]) {
#pragma unroll
  for (int j = 0; j < 16; j++)
    c[j] = (cb + j < N && row >= cb + j) ? p[(int64_t)j * ld] : 0.0f;
}

// One part of a loader's work: 16 panel columns of one row for one operand
// image of one chunk.
struct LPart {
  const float* row_ptr;   // the front's element (row, 0)
  int64_t ld;
  int kc, kend;           // first column of the part, end of the panel
  bool row_ok;            // row < N
  int img, h;             // 0 = tile rows (A), 1 = tile columns (B); half of the chunk
  bool first, last;       // first / last part of its chunk
  uint32_t use;           // how many times the loader's stage was filled before
  __device__ __forceinline__ void load(float (&x)[16]) const {
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const int col = kc + j;
      x[j] = (row_ok && col < kend) ? __ldg(row_ptr + (int64_t)col * ld) : 0.0f;
    }
  }
};

// The parts of loader group q, in order: the chunks g = q, q + NLOAD, ... of
// the CTA's tiles, each 2 or 4 parts.
struct LoaderIter {
  const int* pre;
  int nf;
  const int* flist;
  const FrontDev* fr;
  float* F;
  int K, total, q, t;
  int tile;
  bool have_ti = false;
  TileInfo ti;
  int c = 0, p = 0;
  uint32_t g = 0;
  __device__ LoaderIter(const int* pre_, int nf_, const int* flist_, const FrontDev* fr_, float* F_,
                        int K_, int total_, int q_, int t_)
      : pre(pre_), nf(nf_), flist(flist_), fr(fr_), F(F_), K(K_), total(total_), q(q_), t(t_),
        tile(blockIdx.x) {}
  __device__ bool next(LPart& o) {
    while (true) {
      if (tile >= total) return false;
      if (!have_ti) {
        ti = tile_info(pre, nf, flist, fr, F, K, tile);
        have_ti = true;
        c = 0;
        p = 0;
      }
      if (c >= ti.nch) {
        tile += gridDim.x;
        have_ti = false;
        continue;
      }
      const int nparts = ti.diag ? 2 : 4;
      if ((int)(g % NLOAD) != q || p >= nparts) {
        c++;
        g++;
        p = 0;
        continue;
      }
      o.img = p >> 1;
      o.h = p & 1;
      const int row = (o.img ? ti.c0 : ti.r0) + t;
      o.row_ok = row < ti.N;
      o.row_ptr = ti.A + row;
      o.ld = ti.ld;
      o.kc = K + c * TK + o.h * 16;
      o.kend = ti.k1;
      o.first = p == 0;
      o.last = p == nparts - 1;
      o.use = g / NSTAGE;
      p++;
      return true;
    }
  }
};

// Split 16 values of row t into the hi / lo images of operand `img`, columns
// 16 h .. 16 h + 15 of the chunk.
template <int SPLIT>
__device__ __forceinline__ void store_part(const float (&x)[16], unsigned char* st, int img, int h,
                                           int t) {
  unsigned char* hi = st + img * 2 * IMG;
  unsigned char* lo = hi + IMG;
  const int sw = t & 7;
#pragma unroll
  for (int g4 = 0; g4 < 4; g4++) {
    const int gch = h * 4 + g4;
    float4 hv, lv;
    float* hp = &hv.x;
    float* lp = &lv.x;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float v = x[4 * g4 + e];
      const float vh = tf32_round(v);
      hp[e] = vh;
      if (SPLIT == 3) lp[e] = tf32_round(v - vh);
    }
    const int off = t * 128 + ((gch ^ sw) << 4);
    *reinterpret_cast<float4*>(hi + off) = hv;
    if (SPLIT == 3) *reinterpret_cast<float4*>(lo + off) = lv;
  }
}

template <int SPLIT>
__global__ void __launch_bounds__(TCT, 1) k_trail_tc(const int* __restrict__ flist, int nf,
                                                     const FrontDev* __restrict__ fr,
                                                     float* __restrict__ F, int K, DevError* err) {
  extern __shared__ unsigned char tc_raw[];
  __shared__ uint64_t full[NSTAGE], empty[NSTAGE], acc_full[NACC], acc_empty[NACC];
  __shared__ uint32_t tmem_base;
  __shared__ int pre[kMaxTcFronts + 1];
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* sm =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~(uintptr_t)1023);

  if (tid == 0) {
    int acc = 0;
    pre[0] = 0;
    for (int i = 0; i < nf; i++) {
      const FrontDev d = fr[flist[i]];
      int t = 0;
      if (K < d.n) {
        const int k1 = min(K + kTcOuter, d.n);
        if (d.N > k1) {
          const int T = (d.N - k1 + TM - 1) / TM;
          t = T * (T + 1) / 2;
        }
      }
      acc += t;
      pre[i + 1] = acc;
    }
    for (int s = 0; s < NSTAGE; s++) {
      mbar_init(&full[s], 128);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NACC; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 128);
    }
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

  if (warp < MMA_WARP) {
    // ---- loaders: group q fills stage q with chunks g = q, q + 3, ...; each
    // chunk is 2 (diagonal tile) or 4 parts of 16 columns; the next part's
    // global loads are issued before the current part is converted and before
    // its stage is known to be free, so a thread always has loads in flight ----
    const int q = warp >> 2, t = tid & 127;
    unsigned char* st = sm + q * STAGE_BYTES;
    LoaderIter it(pre, nf, flist, fr, F, K, total, q, t);
    float cur[16], nxt[16];
    LPart pc, pn;
    bool have = it.next(pn);
    if (have) pn.load(nxt);
    while (have && !abort_flag) {
      pc = pn;
#pragma unroll
      for (int j = 0; j < 16; j++) cur[j] = nxt[j];
      have = it.next(pn);
      if (have) pn.load(nxt);
      if (pc.first && pc.use >= 1 && !mbar_wait(&empty[q], (pc.use - 1) & 1, &abort_flag)) break;
      store_part<SPLIT>(cur, st, pc.img, pc.h, t);
      if (pc.last) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(&full[q]);
      }
    }
  } else if (warp == MMA_WARP) {
    // ---- MMA issue ----
    uint32_t g = 0, tl = 0;
    for (int tile = blockIdx.x; tile < total && !__shfl_sync(0xffffffffu, abort_flag, 0);
         tile += gridDim.x, tl++) {
      const TileInfo ti = tile_info(pre, nf, flist, fr, F, K, tile);
      const int b = tl % NACC;
      const uint32_t v = tl / NACC;
      if (v >= 1 && !mbar_wait_warp(&acc_empty[b], (v - 1) & 1, &abort_flag)) break;
      tc_fence_after();
      const uint32_t dacc = tmem + b * TN;
      bool ok = true;
      for (int c = 0; c < ti.nch; c++, g++) {
        const int s = g % NSTAGE;
        if (!mbar_wait_warp(&full[s], (g / NSTAGE) & 1, &abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t a_hi = smem_u32(sm + s * STAGE_BYTES), a_lo = a_hi + IMG;
          const uint32_t b_hi = ti.diag ? a_hi : a_hi + 2 * IMG;
          const uint32_t b_lo = ti.diag ? a_lo : a_hi + 3 * IMG;
#pragma unroll
          for (int kk = 0; kk < TK / 8; kk++) {
            const uint32_t ko = kk * 32;   // 8 TF32 values = 32 bytes along the swizzled row
            mma_tf32(dacc, sw128_desc(a_hi + ko), sw128_desc(b_hi + ko), (c | kk) != 0);
            if (SPLIT == 3) {
              mma_tf32(dacc, sw128_desc(a_hi + ko), sw128_desc(b_lo + ko), 1u);
              mma_tf32(dacc, sw128_desc(a_lo + ko), sw128_desc(b_hi + ko), 1u);
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
  } else {
    // ---- epilogue: C(tile) -= acc ----
    const int quarter = warp & 3;   // tensor-memory lanes this warp may read
    uint32_t tl = 0;
    for (int tile = blockIdx.x; tile < total && !__shfl_sync(0xffffffffu, abort_flag, 0);
         tile += gridDim.x, tl++) {
      const TileInfo ti = tile_info(pre, nf, flist, fr, F, K, tile);
      const int b = tl % NACC;
      const int row = ti.r0 + quarter * 32 + lane;
      const bool live = row < ti.N;
      float* p = ti.A + row + (int64_t)ti.c0 * ti.ld;
      float cur[16];
      if (live) c_load(p, ti.ld, row, ti.c0, ti.N, cur);
      if (!mbar_wait_warp(&acc_full[b], (tl / NACC) & 1, &abort_flag)) break;
      tc_fence_after();
      const uint32_t src = tmem + b * TN + ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
      for (int qb = 0; qb < TN / 16; qb++) {
        uint32_t v[16];
        tmem_ld16(src + qb * 16, v);
        const int cb = ti.c0 + qb * 16;
        float nxt[16];
        if (live && qb + 1 < TN / 16)
          c_load(p + (int64_t)(qb + 1) * 16 * ti.ld, ti.ld, row, cb + 16, ti.N, nxt);
        if (live) {
#pragma unroll
          for (int j = 0; j < 16; j++)
            if (cb + j < ti.N && row >= cb + j)
              p[(int64_t)(qb * 16 + j) * ti.ld] = cur[j] - __uint_as_float(v[j]);
        }
        if (qb + 1 < TN / 16)
#pragma unroll
          for (int j = 0; j < 16; j++) cur[j] = nxt[j];
      }
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

int64_t tc_tiles(const std::vector<int>& n, const std::vector<int>& N, int K) {
  int64_t t = 0;
  for (size_t i = 0; i < n.size(); i++) {
    if (K >= n[i]) continue;
    const int k1 = std::min(K + kTcOuter, n[i]);
    if (N[i] <= k1) continue;
    const int64_t T = (N[i] - k1 + TM - 1) / TM;
    t += T * (T + 1) / 2;
  }
  return t;
}

cudaError_t launch_trail_tc(const int* flist, int nf, int64_t ntiles, const FrontDev* fr, float* F,
                            int K, int split, DevError* err, cudaStream_t st) {
  if (nf <= 0 || ntiles <= 0) return cudaSuccess;
  if (nf > kMaxTcFronts || (split != 1 && split != 3)) return cudaErrorInvalidValue;
  static const int sms = []() {   // thread-safe one-time set-up
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_trail_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    cudaFuncSetAttribute(k_trail_tc<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    return n;
  }();
  const int grid = (int)std::min<int64_t>(ntiles, sms);
  if (split == 3)
    k_trail_tc<3><<<grid, TCT, kTcSmem, st>>>(flist, nf, fr, F, K, err);
  else
    k_trail_tc<1><<<grid, TCT, kTcSmem, st>>>(flist, nf, fr, F, K, err);
  g_launches++;
  return cudaGetLastError();
}

}  // namespace mfgpu
