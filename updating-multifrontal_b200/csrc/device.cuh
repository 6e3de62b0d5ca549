// Device-side tables and kernel entry points shared by the handle code.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

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

// Error word written by kernels: first failing front, column and code.
struct DevError {
  int code;     // 0 ok, 1 non-positive pivot
  int front;
  int col;
  int pad;
};

constexpr int kTaskTile = 32;   // assembly tile edge
constexpr int kPanel = 32;      // panel width of the partial Cholesky

// Assembly tasks: tstart has ntasks+1 exclusive prefix sums of tile counts.
void launch_tasks(const Task* tasks, const int64_t* tstart, int ntasks, int64_t ntiles,
                  double* fronts, double* seps, const int* rp, const int* ci, const double* va,
                  const int* dofs, cudaStream_t st);

// One panel step k of the partial Cholesky for every front in flist: the
// diagonal block factorization, the triangular solve of the rows below it
// (max_rows bounds N - k over the list) and the trailing symmetric update.
void launch_potrf(const int* flist, int nf, const FrontDev* fr, double* F, int k, DevError* err,
                  cudaStream_t st);
void launch_trsm(const int* flist, int nf, const FrontDev* fr, double* F, int k, int max_rows,
                 cudaStream_t st);
void launch_syrk(const int* flist, int nf, const FrontDev* fr, double* F, int k, int max_rows,
                 cudaStream_t st);

// Fused partial factorization of every front in flist, one CTA per front
// (fronts with n + m <= 640; small_front_fits tells).
bool small_front_fits(int maxN);
void launch_front_small(const int* flist, int nf, int maxN, const FrontDev* fr, double* F,
                        DevError* err, cudaStream_t st);

// Partial factorization of every front in flist (at most 256 fronts) by one
// cooperative persistent launch over all SMs.
// `slots` holds coop_slot_doubles() doubles of device scratch.
bool coop_fits(int nf);
size_t coop_slot_doubles();
cudaError_t launch_level_coop(const int* flist, int nf, int maxn, const FrontDev* fr, double* F,
                              DevError* err, double* slots, cudaStream_t st);

// Number of kernels this library has launched since it was loaded.
long long launches_total();

// Solve / apply sweeps (nrhs <= 16 per call).  W holds 2*N*nrhs doubles per
// front at offset woff[f]*nrhs (woff = exclusive prefix of 2*N).
void launch_solve_fwd(const int* flist, int nf, int maxN, const FrontDev* fr, const double* F,
                      const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                      const int64_t* woff, cudaStream_t st);
void launch_solve_bwd(const int* flist, int nf, int maxN, const FrontDev* fr, const double* F,
                      const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                      const int64_t* woff, cudaStream_t st);
void launch_sep_gather(const int* slist, int ns, const SepDev* sp, const int* dofs, double* X,
                       int64_t ldx, int nrhs, const double* W, const int64_t* woff,
                       const FrontDev* fr, cudaStream_t st);
void launch_apply_up(const int* flist, int nf, const FrontDev* fr, const double* F,
                     const int* dofs, double* X, int64_t ldx, int nrhs, double* W,
                     const int64_t* woff, double* T, cudaStream_t st);
void launch_apply_down(const int* flist, int nf, const FrontDev* fr, const double* F,
                       const int* dofs, int64_t ldx, int nrhs, double* W, const int64_t* woff,
                       const double* T, cudaStream_t st);
void launch_root_solve(int f, int N, const FrontDev* fr, const double* F, const int* dofs,
                       double* X, int64_t ldx, int nrhs, double* W, const int64_t* woff,
                       cudaStream_t st);
void launch_root_apply(int f, const FrontDev* fr, const double* F, const int* dofs, double* X,
                       int64_t ldx, int nrhs, double* W, const int64_t* woff, cudaStream_t st);

}  // namespace mfgpu
