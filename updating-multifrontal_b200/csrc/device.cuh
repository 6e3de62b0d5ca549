// Device-side tables and kernel entry points shared by the handle code.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "schedule.hpp"

namespace mfgpu {

// Compact per-front descriptor read by every kernel.
struct FrontDev {
  int64_t off;      // element offset of the front (column-major, ld) in the arena
  int64_t dof_off;  // offset of [pivots..., boundary...] in the DOF table
  int n, m, N, ld;
};
static_assert(sizeof(FrontDev) == 32, "FrontDev layout");

// Per-separator descriptor for the solve/apply gathers.
struct SepDev {
  int64_t dof_off;
  int s;
  int box0, box1;      // global front ids (reference order: box0 then box1)
  int pos0, pos1;      // row of the separator inside each box's front
  int pad;
};
static_assert(sizeof(SepDev) == 32, "SepDev layout");

// Error word written by kernels: first failing front, column and code.  The
// host also places the poll limit of the bounded waits in it (0: the built-in
// limits), so a launch reads the limit from the word it reports into.
struct DevError {
  int code;        // 0 ok, 1 non-positive pivot, 2 tensor-core wait, 3 grid barrier timed out,
                   // 4 zero pivot column of an LU front
  int front;
  int col;
  unsigned limit;  // polls before a bounded wait gives up; 0 = the built-in limit
};
static_assert(sizeof(DevError) == 16, "DevError layout");

// Poll limit of a bounded wait: the host-set one from the error word, else dflt.
__device__ __forceinline__ unsigned wait_limit(const DevError* err, unsigned dflt) {
  if (!err) return dflt;
  const unsigned l = *reinterpret_cast<const volatile unsigned*>(&err->limit);
  return l ? l : dflt;
}

// Grid-wide barrier of the cooperative kernels, with a bounded wait.  `count`
// (one unsigned per launch, zeroed before the launch on the launch's stream)
// counts arrivals; `target` is private to each thread and advances by the grid
// size at every barrier.  A wait that gives up (after the error word's poll
// limit, default kBarrierSpin) records error code 3 in the error word; every
// later barrier of any CTA then passes at once, so the launch always ends.
// The fences follow the usual grid-barrier pattern: the CTA's writes are
// ordered before thread 0's arrival, and thread 0's observation of the last
// arrival before the CTA's later reads.
constexpr unsigned kBarrierSpin = 1u << 25;
__device__ __forceinline__ void grid_barrier(unsigned* count, unsigned& target, DevError* err) {
  __syncthreads();
  target += gridDim.x;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    __threadfence();
    atomicAdd(count, 1u);
    volatile unsigned* c = count;
    volatile int* code = err ? &err->code : nullptr;
    const unsigned lim = wait_limit(err, kBarrierSpin);
    unsigned it = 0;
    while (*c < target) {
      if (++it > lim) {
        if (err) atomicCAS(&err->code, 0, 3);
        break;
      }
      if ((it & 1023u) == 0 && code && *code == 3) break;   // another CTA gave up
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
}

constexpr int kTaskTile = 32;   // assembly tile edge
constexpr int kPanel = 32;      // panel width of the partial Cholesky

// Kernel launch wrappers.  T = double (FP64 path) or float (mixed path).

// Assembly tasks: tstart has ntasks+1 exclusive prefix sums of tile counts.
// `scale` (may be null) multiplies sparse entries a_rc by scale[r] * scale[c].
template <class T>
void launch_tasks(const Task* tasks, const int64_t* tstart, int ntasks, int64_t ntiles, T* fronts,
                  T* seps, const int* rp, const int* ci, const double* va, const int* dofs,
                  const double* scale, cudaStream_t st);

// Stepped FP64 path (one launch per panel step and kernel), kept for levels a
// cooperative launch cannot take.
void launch_potrf(const int* flist, int nf, const FrontDev* fr, double* F, int k, DevError* err,
                  cudaStream_t st);
void launch_trsm(const int* flist, int nf, const FrontDev* fr, double* F, int k, int max_rows,
                 cudaStream_t st);
void launch_syrk(const int* flist, int nf, const FrontDev* fr, double* F, int k, int max_rows,
                 cudaStream_t st);

// Fused partial factorization, one CTA per front, for levels whose widest
// front's staged panel fits in shared memory.
bool small_front_fits(int maxN, int elem_bytes);
template <class T>
void launch_front_small(const int* flist, int nf, int maxN, const FrontDev* fr, T* F, DevError* err,
                        cudaStream_t st);

// Partial factorization of every front in flist by one cooperative persistent
// launch over all SMs.  `slots` holds coop_slot_elems() elements of scratch;
// `phase_pref` the per-phase work-item prefixes from coop_phase_prefix.
bool coop_fits(int nf);
size_t coop_slot_elems();
std::vector<int> coop_phase_prefix(const std::vector<int>& n, const std::vector<int>& N, int maxn,
                                   int outer = 0);
// max_items (> 0): the largest work-item count of any phase, to size the grid;
// K0/K1/phase0/trailing restrict the launch to the outer panels [K0, K1)
// (K1 < 0: to the end) and optionally leave the last trailing update out;
// outer (> 0) is the outer panel width, a multiple of 32 (default
// coop_outer()), and must match the one phase_pref was built with.
// gbar: one unsigned of device memory for the launch's grid barrier.
template <class T>
cudaError_t launch_level_coop(const int* flist, int nf, int maxn, const FrontDev* fr, T* F,
                              DevError* err, T* slots, const int* phase_pref, unsigned* gbar,
                              cudaStream_t st, int K0 = 0, int K1 = -1, int phase0 = 0,
                              int trailing = 1, int max_items = 0, int outer = 0);
int coop_outer();   // default outer panel width of the cooperative kernel
// phases of outer panel K in the prefix table built with this outer width
int coop_phases(int K, int maxn, int outer = 0);

// Tensor-core (tcgen05, TF32) trailing update of the mixed path after outer
// panel K of every front in flist: C(k1:N, k1:N) -= P P^T with P the panel's
// columns, split = 1 (TF32) or 3 (hi/lo three-term TF32, about FP32 accuracy).
// launch_tc_pack first writes P, split into TF32 hi / lo tensor-core images,
// into `pack` (tc_pack_bytes(nf, cap) bytes, cap = tc_pack_cap(n, N, K, w));
// launch_trail_tc then reads P only from there.
int tc_outer();
int tc_max_fronts();
// The panel is [K, K + w) (w a multiple of 32, at most tc_outer()); the
// update covers columns below cend (cend < 0: all columns, else
// min(cend, n) per front).
int64_t tc_tiles(const std::vector<int>& n, const std::vector<int>& N, int K, int w, int cend);
int tc_pack_cap(const std::vector<int>& n, const std::vector<int>& N, int K, int w);
size_t tc_pack_bytes(int nf, int cap);
cudaError_t launch_tc_pack(const int* flist, int nf, int cap, const FrontDev* fr, const float* F,
                           int K, int w, int split, void* pack, cudaStream_t st);
// Panel-by-panel partial Cholesky without grid barriers (kernels_panel.cu):
// launch_subpanel turns the panel [Ks, Ks + w) of every front in flist into L
// (w = panel_width(sizeof(T)): 64 FP64, 128 FP32; every earlier update
// applied), launch_trail_syrk applies it to the trailing lower triangle.  At
// most kMaxPanelFronts fronts per launch; dslot: panel_slot_bytes(nf, sizeof(T))
// of scratch for the inverses of the factored diagonal blocks.
constexpr int kPanelW64 = 64, kPanelW32 = 128, kMaxPanelFronts = 1024;
int panel_width(int elem_bytes);
size_t panel_slot_bytes(int nf, int elem_bytes);
template <class T>
cudaError_t launch_subpanel(const int* flist, int nf, const FrontDev* fr, T* F, int Ks, int w,
                            T* dslot, DevError* err, cudaStream_t st);
template <class T>
cudaError_t launch_trail_syrk(const int* flist, int nf, const FrontDev* fr, T* F, int Ks, int w,
                              cudaStream_t st);
cudaError_t launch_trail_tc(const int* flist, int nf, int64_t ntiles, const FrontDev* fr, float* F,
                            int K, int w, int cend, int split, int cap, const void* pack,
                            DevError* err, cudaStream_t st);

// Cooperative sweeps over all fronts of one level (nrhs <= 16), ordered by
// ready flags instead of grid barriers: forward = L11 solve and boundary update
// b_bd -= L21 y, backward = L21^T update and L11^T solve, both gathering from
// and scattering to X themselves.  flow_tasks builds a level's task lists
// (front slot, block) pairs, forward R-major and backward by distance from
// each front's last block, and the per-front offsets of the ready flags
// (flagoff[nf] = flags needed); `flags` is cleared before every launch.
int solve_coop_max_fronts();
void flow_tasks(const std::vector<int>& n, const std::vector<int>& N, std::vector<int>& fwd,
                std::vector<int>& bwd, std::vector<int>& flagoff);
// The sweeps apply each 64 x 64 pivot block through its explicit inverse (Dv,
// per front at dinv_off, written by launch_diag_inv after the front is
// factored) and keep solved blocks in the second half of the front's
// workspace, where other tasks read them.
template <class T>
cudaError_t launch_solve_flow(bool forward, const int* flist, const FrontDev* fr, const T* F,
                              const int* dofs, T* X, int64_t ldx, int nrhs, T* W,
                              const int64_t* woff, const T* Dv, const int64_t* dinv_off,
                              const int* tasks, int ntasks, const int* flagoff, int* flags,
                              int nflags, DevError* err, cudaStream_t st);
constexpr int kDinvBlock = 64;   // diagonal-block size of the cooperative sweeps
template <class T>
void launch_diag_inv(const int* flist, int nf, int maxn, const FrontDev* fr, const T* F, T* Dv,
                     const int64_t* dinv_off, cudaStream_t st);

// Pivoted LU of nonsymmetric fronts (separator width 2-3), FP64
// (kernels_lu.cu).  One 32-column step k of every front in flist: phase 0
// factors the panel (pivots among the pivot rows, recorded in ipiv at the
// front's DOF offset), phase 1 applies its row swaps to the other columns and
// solves the block row, phase 2 updates the trailing matrix.  maxN: the
// level's largest front.
void launch_lu_step(const int* flist, int nf, int maxN, const FrontDev* fr, double* F, int* ipiv,
                    int k, DevError* err, cudaStream_t st, int phase);
// Sweeps of LU fronts (nrhs <= 16): forward = gather, row swaps, unit-L11
// solve and boundary update; backward = gather, U12 update and U11 solve.
void launch_lu_solve(bool forward, const int* flist, int nf, int maxN, const FrontDev* fr,
                     const double* F, const int* ipiv, const int* dofs, double* X, int64_t ldx,
                     int nrhs, double* W, const int64_t* woff, cudaStream_t st);
// Apply, upward part, of LU fronts (the downward part is launch_apply_down).
void launch_lu_apply_up(const int* flist, int nf, const FrontDev* fr, const double* F,
                        const int* ipiv, const int* dofs, double* X, int64_t ldx, int nrhs,
                        double* W, const int64_t* woff, double* Tb, cudaStream_t st);

// Stencil assembly (width 1): recompute the CSR values of the rows of the
// cells in [lo, hi) from the node coefficients; with `flag`, record which rows
// changed; launch_collect_rows appends the flagged rows to `out`.
cudaError_t launch_stencil_rows(int dim, int nx, int ny, int nz, const double h[3], const double* a,
                                const int* rp, double* val, const int lo[3], const int hi[3],
                                int* flag, cudaStream_t st);
cudaError_t launch_collect_rows(int dim, int nx, int ny, const int lo[3], const int hi[3],
                                const int* flag, int* out, int cap, int* count, cudaStream_t st);
// Node coefficients of the cells [lo, hi) multiplied by factor (in place).
cudaError_t launch_scale_box(int dim, int ny, int nz, const int lo[3], const int hi[3], double factor,
                             double* a, cudaStream_t st);

// Number of kernels this library has launched since it was loaded.
long long launches_total();

// Solve / apply sweeps (nrhs <= 16 per call).  W holds 2*N*nrhs elements per
// front at offset woff[f]*nrhs (woff = exclusive prefix of 2*N).
template <class T>
void launch_solve_fwd(const int* flist, int nf, int maxN, const FrontDev* fr, const T* F,
                      const int* dofs, T* X, int64_t ldx, int nrhs, T* W, const int64_t* woff,
                      cudaStream_t st);
template <class T>
void launch_solve_bwd(const int* flist, int nf, int maxN, const FrontDev* fr, const T* F,
                      const int* dofs, T* X, int64_t ldx, int nrhs, T* W, const int64_t* woff,
                      cudaStream_t st);
template <class T>
void launch_root_solve(int f, int N, const FrontDev* fr, const T* F, const int* dofs, T* X,
                       int64_t ldx, int nrhs, T* W, const int64_t* woff, cudaStream_t st);
template <class T>
void launch_sep_gather(const int* slist, int ns, const SepDev* sp, const int* dofs, T* X,
                       int64_t ldx, int nrhs, const T* W, const int64_t* woff, const FrontDev* fr,
                       cudaStream_t st);
template <class T>
void launch_apply_up(const int* flist, int nf, const FrontDev* fr, const T* F, const int* dofs, T* X,
                     int64_t ldx, int nrhs, T* W, const int64_t* woff, T* Tb, cudaStream_t st);
template <class T>
void launch_apply_down(const int* flist, int nf, const FrontDev* fr, const T* F, const int* dofs,
                       int64_t ldx, int nrhs, T* W, const int64_t* woff, const T* Tb,
                       cudaStream_t st);
template <class T>
void launch_root_apply(int f, const FrontDev* fr, const T* F, const int* dofs, T* X, int64_t ldx,
                       int nrhs, T* W, const int64_t* woff, cudaStream_t st);

// Vector kernels of the mixed-precision solve (kernels_vec.cu).
void launch_diag_scale(const int* rp, const int* ci, const double* va, int n, double* s,
                       double* is, cudaStream_t st);
void launch_spmv(const int* rp, const int* ci, const double* va, int n, const double* x, int64_t ldx,
                 double* y, int64_t ldy, int nrhs, cudaStream_t st);
void launch_residual(const int* rp, const int* ci, const double* va, int n, const double* b,
                     int64_t ldb, const double* x, int64_t ldx, double* r, int64_t ldr, int nrhs,
                     cudaStream_t st);
// Segmented deterministic dots: dot_plan cuts each segment [seg_row[g],
// seg_row[g+1]) into fixed chunks; launch_dot writes out[g + nseg * c].
void dot_plan(const std::vector<int64_t>& seg_row, std::vector<int>& chunk_row,
              std::vector<int>& seg_chunk);
void launch_dot(const double* x, int64_t ldx, const double* y, int64_t ldy, int nrhs,
                const int* chunk_row, int nchunks, const int* seg_chunk, int nseg, double* part,
                double* out, cudaStream_t st);
template <class T>
void launch_scale_to(const double* src, int64_t lds, T* dst, int64_t ldd, const double* s, int n,
                     int nrhs, cudaStream_t st);
template <class T>
void launch_scale_from(const T* src, int64_t lds, double* dst, int64_t ldd, const double* s, int n,
                       int nrhs, cudaStream_t st);
// PCG updates with per-(segment, column) scalars; seg_row holds the nseg + 1
// segment boundaries (rows) on the device.
void launch_pcg_xr(double* x, double* r, const double* p, const double* q, int64_t ld, int n,
                   int nrhs, const double* rz, const double* pq, const int* active,
                   const int* seg_row, int nseg, cudaStream_t st);
void launch_pcg_p(double* p, const double* z, int64_t ld, int n, int nrhs, const double* rz_new,
                  const double* rz_old, const int* active, int first, const int* seg_row, int nseg,
                  cudaStream_t st);

}  // namespace mfgpu
