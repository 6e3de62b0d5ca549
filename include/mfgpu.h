/*
 * mfgpu.h — C ABI of the B200 multifrontal factor / localized-update / solve
 * path for box/separator-ordered 2D 5-point and 3D 7-point variable-coefficient
 * Laplacians.
 *
 * Every entry point takes plain pointers and sizes.  Each one replaces a public
 * member of the reference's TreeFactor2D::MF2D<double> / TreeFactor3D::MF3D<double>
 * (victorminden/updating-multifrontal, include/DE/mf.hpp); the citation is
 * given beside each declaration.  Errors are reported as status codes; the
 * C++ drop-in headers turn them back into the reference's exceptions.
 *
 * A handle owns its device memory (CSR matrix, symbolic tables, factor,
 * update matrices) and one CUDA stream; the factorization stays resident on
 * the GPU between calls.  One handle must be used by one host thread at a
 * time.  There is no CPU fallback: without a usable CUDA device every
 * compute call fails with MFGPU_ERR_CUDA.
 */
#ifndef MFGPU_H
#define MFGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mfgpu_handle mfgpu_handle;
typedef struct mfgpu_symbolic mfgpu_symbolic;
typedef struct mfgpu_server mfgpu_server;

enum mfgpu_status {
  MFGPU_OK = 0,
  MFGPU_ERR_ARG = 1,        /* bad argument (sizes, null pointers, pattern)  */
  MFGPU_ERR_DEPTH = 2,      /* tree depth <= 1 (reference: runtime_error)    */
  MFGPU_ERR_LEAF = 3,       /* leaf-width arithmetic failed (runtime_error)  */
  MFGPU_ERR_OOM = 4,        /* device allocation failed                      */
  MFGPU_ERR_CUDA = 5,       /* CUDA runtime error or no device               */
  MFGPU_ERR_PIVOT = 6,      /* non-positive pivot: matrix not SPD            */
  MFGPU_ERR_TIMEOUT = 7,    /* a bounded device wait gave up                 */
  MFGPU_ERR_STATE = 8,      /* call out of order (e.g. solve before factor)  */
  MFGPU_ERR_NOT_CONVERGED = 9 /* mixed precision: refinement did not reach tol */
};

enum mfgpu_precision {
  MFGPU_FP64 = 0,   /* drop-in path: FP64 factor and solve                    */
  MFGPU_MIXED = 1   /* FP32/tensor-core factor, FP64 residual + refinement    */
};

typedef struct mfgpu_options {
  int precision;        /* mfgpu_precision, default MFGPU_FP64                  */
  int device;           /* CUDA device ordinal, default 0                       */
  double refine_tol;    /* mixed: target ||b-Ax||/||b||, default 1e-10          */
  int refine_maxit;     /* mixed: refinement iteration cap, default 50          */
  int reserved[7];
} mfgpu_options;

typedef struct mfgpu_info {
  int dim, levels, n_fronts, n_seps;
  int64_t ndof, nnz;
  int leaf_box[3];              /* leaf box widths (boxWidth{X,Y,Z}Bottom_)   */
  int max_front;                /* largest n + m                              */
  double factor_flops;          /* sum over fronts of n^3/3 + n^2 m + n m^2   */
  int64_t front_bytes, sep_bytes, device_bytes;
} mfgpu_info;

typedef struct mfgpu_stats {
  double seconds;         /* device time of the last factor/update/solve call */
  double flops;           /* algorithmic flops of that call (Cholesky form)   */
  int fronts;             /* fronts (boxes) refactored by the last factor/update */
  int iterations;         /* refinement iterations of the last mixed solve    */
  double residual;        /* last mixed solve: max_j ||b_j - A x_j|| / ||b_j|| */
} mfgpu_stats;

void mfgpu_default_options(mfgpu_options* opts);
const char* mfgpu_status_string(int status);

/* MF2D(const Sparse&, Nx, Ny, width, maxSideLength) — include/DE/mf.hpp:74;
 * MF3D(const Sparse&, Nx, Ny, Nz, width, maxSideLength) — include/DE/mf.hpp:180.
 * dim = 2 ignores nz.  The CSR (row_ptr[n+1], col_ind[nnz], val[nnz]) is copied.
 * width = 1 (5-/7-point stencils): the matrix must be symmetric positive
 * definite and is factored by Cholesky; one that is not symmetric (to a
 * relative 1e-12) is refused with MFGPU_ERR_ARG, naming the first unequal
 * pair; indefiniteness surfaces as MFGPU_ERR_PIVOT in the factorization.
 * width = 2 or 3 (the reference fixture's wider stencils, nonsymmetric with
 * variable coefficients): every front is factored by LU with partial pivoting
 * inside its pivot block, as the reference's dgetrf on A22
 * (include/LinAlg/dense.hpp:180-227); FP64 only (MFGPU_ERR_ARG otherwise), no
 * batches, serving loop or autotuner; a singular pivot block surfaces as
 * MFGPU_ERR_PIVOT. */
int mfgpu_create(int dim, int nx, int ny, int nz, int width, int max_side_length, int n,
                 const int* row_ptr, const int* col_ind, const double* val,
                 const mfgpu_options* opts, mfgpu_handle** out);

/* Stencil assembly on the device (no reference counterpart; restates the
 * reference fixture test_include/DE/buildLaplacian.hpp:10-132, 244-391 for
 * width 1, bit for bit).  d_coef: node coefficients, (nx+2) x (ny+2)
 * [x (nz+2)] doubles, C order with x slowest; hxyz: grid spacings (null = 1).
 * Writes every CSR value of the handle's pattern into d_val (nnz doubles). */
int mfgpu_stencil_assemble_device(mfgpu_handle* h, const double* d_coef, const double* hxyz,
                                  double* d_val);

/* After the coefficients of the cells in the box [box_lo, box_hi) changed
 * (d_coef holds the new array), recompute the affected rows of d_val in place
 * and return the modified DOFs (rows with a changed entry, sorted: the set the
 * reference's test computes on the host, test_src/DE/testMF2D.cpp:143-150),
 * ready for mfgpu_update_device. */
int mfgpu_stencil_update_device(mfgpu_handle* h, const double* d_coef, const double* hxyz,
                                const int* box_lo, const int* box_hi, double* d_val,
                                int* modified_dofs, int capacity, int* n_modified);

/* ---- Update-serving loop (no reference counterpart) ----
 * A factored handle stays resident; each request multiplies the coefficients
 * of one box of cells [box_lo, box_hi) by `factor` and solves the changed
 * system for its right-hand sides.  Requests are independent of each other
 * (each answer is that of the base matrix under its own change) and refactor
 * only the root paths of the leaves their box touches (the reference's
 * Update, src/DE/mf2d.cpp:150-181) into private copies held in a device pool
 * of pool_bytes.  Continuous batching: one dispatcher takes queued requests in
 * arrival order into a batch of at most `slots` requests whose private copies
 * fit in the pool together, refactors all their root paths with one set of
 * level launches (their overlapping paths - every path reaches the root - are
 * factored side by side in the same launches), solves each, and meanwhile
 * arriving requests wait for the next batch.  An answer is bit-identical
 * whether its request ran alone or in a batch.  A request whose private
 * copies exceed the whole pool fails with MFGPU_ERR_OOM.
 * d_coef: the base coefficients on the device ((nx+2) x (ny+2) [x (nz+2)],
 * C order, x slowest), copied by the server; hxyz: grid spacings (null = 1). */
typedef struct mfgpu_request_info {
  int status;               /* mfgpu_status of the request                       */
  int fronts;               /* fronts refactored for it                          */
  int iterations;           /* refinement iterations (mixed)                     */
  int batch;                /* requests served in its batch (itself included)    */
  double queued_seconds;    /* submit -> start of its batch                      */
  double latency_seconds;   /* submit -> result written                          */
  double residual;          /* relative residual reached (mixed)                 */
  int64_t pool_bytes;       /* private memory it held                            */
  int64_t reserved[4];
} mfgpu_request_info;

int mfgpu_server_create(mfgpu_handle* base, const double* d_coef, const double* hxyz, int slots,
                        int64_t pool_bytes, mfgpu_server** out);
/* Queue a request (host b, nrhs columns of leading dimension ld >= n); the
 * answer is written to host x (same ld) before mfgpu_server_wait returns. */
int mfgpu_server_submit(mfgpu_server* srv, const int* box_lo, const int* box_hi, double factor,
                        const double* b, int nrhs, int64_t ld, double* x, int64_t* ticket);
/* Block until the request is done; returns its status (each ticket once). */
int mfgpu_server_wait(mfgpu_server* srv, int64_t ticket, mfgpu_request_info* info);
const char* mfgpu_server_last_error(const mfgpu_server* srv);
void mfgpu_server_destroy(mfgpu_server* srv);

/* Batch of independent problems in one handle (no reference counterpart; the
 * reference factors one problem per MF2D/MF3D object).  Problem p has the
 * geometry (dim[p], nx[p], ny[p], nz[p], width[p], max_side[p]); the matrix is
 * the block-diagonal CSR of the problems (n = sum of their DOFs, global column
 * indices), problem p owning rows offs[p] .. offs[p+1]-1 (mfgpu_batch_info).
 * Every tree level of every problem is factored and solved by the same
 * launches (levels aligned at the leaves).  All other calls work on the
 * stacked vectors; mixed-precision refinement, its scalars and its tolerance
 * are per problem and per right-hand side. */
int mfgpu_batch_create(int count, const int* dim, const int* nx, const int* ny, const int* nz,
                       const int* width, const int* max_side, int n, const int* row_ptr,
                       const int* col_ind, const double* val, const mfgpu_options* opts,
                       mfgpu_handle** out);

/* Number of problems in the handle (1 for mfgpu_create) and, when dof_offsets
 * is not null, their count + 1 row offsets. */
int mfgpu_batch_info(const mfgpu_handle* h, int* count, int64_t* dof_offsets);

/* void Factor() — include/DE/mf.hpp:84, src/DE/mf2d.cpp:449-500. */
int mfgpu_factor(mfgpu_handle* h);

/* void Update(const Sparse& A, std::set<int> modifiedDOFs) — include/DE/mf.hpp:86,
 * src/DE/mf2d.cpp:150-181.  `val` holds the new values on the unchanged pattern
 * (nnz entries); only fronts on root paths of leaves holding modified DOFs are
 * refactored. */
int mfgpu_update(mfgpu_handle* h, const double* val, int64_t nnz, const int* modified_dofs,
                 int n_modified);

/* Device-pointer form of Update (no reference counterpart): d_val in device
 * memory, modified_dofs on the host. */
int mfgpu_update_device(mfgpu_handle* h, const double* d_val, int64_t nnz,
                        const int* modified_dofs, int n_modified);

/* Replace all matrix values (same pattern) and refactor every front: the
 * reference's Update(A, every DOF) (src/DE/mf2d.cpp:150-181 with all leaves
 * marked), without building the modified-DOF set. */
int mfgpu_refactor(mfgpu_handle* h, const double* val, int64_t nnz);
int mfgpu_refactor_device(mfgpu_handle* h, const double* d_val, int64_t nnz);

/* Vec Solve(const Vec& b) — include/DE/mf.hpp:81, src/DE/mf2d.cpp:976-1054.
 * Host buffers: b and x are n x nrhs column-major with leading dimension ld. */
int mfgpu_solve(mfgpu_handle* h, const double* b, double* x, int nrhs, int64_t ld);

/* Vec Apply(const Vec& x) — include/DE/mf.hpp:78, src/DE/mf2d.cpp:904-974. */
int mfgpu_apply(mfgpu_handle* h, const double* x, double* b, int nrhs, int64_t ld);

/* Device-pointer forms of Solve / Apply (no reference counterpart: the
 * reference is host-only); b/x live in device memory. */
int mfgpu_solve_device(mfgpu_handle* h, const double* d_b, double* d_x, int nrhs, int64_t ld);
int mfgpu_apply_device(mfgpu_handle* h, const double* d_x, double* d_b, int nrhs, int64_t ld);

/* Solve with device buffers and no device allocation (no counterpart in the
 * reference, which is host-only).  mfgpu_solve_device grows its workspace with
 * cudaMalloc when it first sees a problem or a larger right-hand-side count;
 * callers that may not allocate at solve time — a service that reserves all
 * device memory at start-up and must stay inside that budget, or a real-time
 * loop that cannot take cudaMalloc's implicit device-wide synchronisation —
 * call this instead.  Its workspace is a fixed 32 MiB array compiled into the
 * library, present on every GPU that loads it until the process exits.
 *   - Problems whose workspace for one right-hand side exceeds 32 MiB are
 *     rejected with MFGPU_ERR_ARG and a message giving the sizes; larger nrhs
 *     is processed in chunks that fit.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call
 *     before any stream capture.
 *   - Every call, from every handle on the device, shares the array and leaves
 *     its last contents in it; calls that overlap on the GPU (other streams,
 *     other threads) race on it and must be serialised by the caller.
 * d_b and d_x are n x nrhs column-major with leading dimension ld in device
 * memory; d_x may equal d_b (in-place).  Returns after the solve completes. */
int mfgpu_solve_device_noalloc(mfgpu_handle* h, const double* d_b, double* d_x, int nrhs,
                               int64_t ld);

/* Use an external CUDA stream (cudaStream_t) for all later work; NULL restores
 * the handle's own stream. */
int mfgpu_set_stream(mfgpu_handle* h, void* cuda_stream);

/* CUDA graphs (no reference counterpart).  A handle replays the launches of
 * its full factorization (every level's assembly, partial factorization and
 * separator accumulation: the level schedule) as one captured CUDA graph from
 * the second full factorization on, and likewise the solve sweeps (FP64) or
 * the preconditioner applications of the refinement (mixed) per right-hand-
 * side buffer and count from their second use; localized updates, whose fronts
 * change from call to call, and the no-allocation solve launch directly.
 * Results are bit-identical either way.  MFGPU_GRAPHS=0 in the environment at
 * creation turns graphs off.  mfgpu_graphs reports whether the factorization
 * graph exists and how many sweep graphs are held. */
int mfgpu_graphs(const mfgpu_handle* h, int* factor_graph, int* sweep_graphs);

/* Failure handling (no reference counterpart: the reference has no device
 * waits, and its LAPACK failures abort through assert, include/LinAlg/dense.hpp:187).
 * Every device wait of this library is bounded: the grid barriers of the
 * cooperative kernels give up after 2^25 polls, the tensor-core pipeline's
 * mbarrier waits after 2^24; a wait that gives up makes the call return
 * MFGPU_ERR_TIMEOUT, and the handle stays usable (the next call starts from a
 * clean error word and barrier counter; refactor before solving again if the
 * timeout hit a factorization).  mfgpu_set_wait_limit sets the poll limit of
 * this handle's later launches (0 restores the built-in limits); serving-loop
 * views created afterwards inherit it.  Waits that drain work already in
 * flight before a kernel exits keep the built-in limit. */
int mfgpu_set_wait_limit(mfgpu_handle* h, unsigned polls);
/* Host-side fault injection for tests: the next `after` device allocations of
 * the library succeed and the one after fails as if the device were out of
 * memory (the call returns MFGPU_ERR_OOM), then injection disarms itself.
 * after < 0 disarms it. */
void mfgpu_inject_alloc_failure(long long after);

/* Factor serialisation (no counterpart in the reference, whose factorization
 * lives in process memory only; use: restart a serving loop without
 * refactoring its base).  mfgpu_save writes a factored handle's state - front
 * and separator arenas, CSR values, the mixed path's scaling, the cooperative
 * sweeps' block inverses - to `path` with a header describing the problem and
 * a checksum of the payload.  mfgpu_load restores it into a handle created
 * for the same problem (same schedule sizes, precision and sparsity pattern);
 * the handle is then factored: Solve, Apply and Update need no Factor().  A
 * file that does not match the handle, or whose checksum fails, is rejected
 * with MFGPU_ERR_ARG (after a failed checksum the handle is left unfactored).
 * Saving an unfactored handle returns MFGPU_ERR_STATE.  Not for the serving
 * loop's per-slot views. */
int mfgpu_save(mfgpu_handle* h, const char* path);
int mfgpu_load(mfgpu_handle* h, const char* path);

/* Autotuner (no counterpart in the reference): a full factorization, like
 * mfgpu_factor, that also picks each tree level's kernel by timing.  For every
 * level with more than one eligible kernel - one CTA per front
 * (MFGPU_LEVEL_FUSED), the cooperative level kernel (MFGPU_LEVEL_COOP),
 * panel-by-panel launches without grid barriers (MFGPU_LEVEL_PANEL), the
 * tensor-core update (MFGPU_LEVEL_TC, mixed precision) - each candidate runs
 * `reps` times on freshly assembled fronts and the fastest is kept; later
 * full factorizations (mfgpu_factor / mfgpu_refactor*) use the table, localized
 * updates keep the size rules (their levels hold far fewer fronts).
 * `choices` (may be NULL) receives the kernel of each level, root = 0,
 * mfgpu_get_info().levels entries. */
enum { MFGPU_LEVEL_NONE = -1, MFGPU_LEVEL_FUSED = 0, MFGPU_LEVEL_COOP = 1, MFGPU_LEVEL_TC = 2,
       MFGPU_LEVEL_STEPPED = 3, MFGPU_LEVEL_LU = 4, MFGPU_LEVEL_PANEL = 5 };
int mfgpu_autotune(mfgpu_handle* h, int reps, int* choices);

/* Per-kernel-class device timing (no reference counterpart; the reference's
 * HASCPP11TIMING millisecond counters, src/DE/mf2d.cpp:15-18, 464-499, are the
 * closest).  When enabled, every launch group is bracketed by CUDA events on
 * the handle's stream; reads return cumulative launches, milliseconds and the
 * algorithmic flops / bytes of the work those launches did. */
enum mfgpu_kernel_class {
  MFGPU_KC_ASSEMBLE = 0,  /* front / separator assembly and accumulation     */
  MFGPU_KC_POTRF = 1,     /* diagonal-block Cholesky of each panel           */
  MFGPU_KC_TRSM = 2,      /* panel triangular solves                         */
  MFGPU_KC_SYRK = 3,      /* trailing symmetric updates (Schur complements)  */
  MFGPU_KC_SOLVE = 4,     /* forward / backward sweeps                       */
  MFGPU_KC_APPLY = 5,     /* factored-operator application                   */
  MFGPU_KC_FRONT = 6,     /* fused partial factorization, one CTA per front  */
  MFGPU_KC_COOP = 7,      /* per-level partial factorization on CUDA cores:
                             cooperative kernel, panel kernels, and the
                             tensor-core levels' sub-panels                   */
  MFGPU_KC_TC = 8,        /* tensor-core trailing updates (mixed path)       */
  MFGPU_KC_COUNT = 9
};
int mfgpu_profile_enable(mfgpu_handle* h, int on);
int mfgpu_profile_reset(mfgpu_handle* h);
int mfgpu_profile_read(const mfgpu_handle* h, int kernel_class, int64_t* launches, double* ms,
                       double* flops, double* bytes);
/* Kernels launched by this library since it was loaded (all handles). */
long long mfgpu_kernel_launches(void);

int mfgpu_get_info(const mfgpu_handle* h, mfgpu_info* info);
int mfgpu_last_stats(const mfgpu_handle* h, mfgpu_stats* stats);
const char* mfgpu_last_error(const mfgpu_handle* h);
void mfgpu_destroy(mfgpu_handle* h);

/* Host-only symbolic schedule (no device needed): the reference's per-level
 * DOF lists (Box::intDOFs / bdDOFs and Edge/Face::DOFs, include/DE/mf.hpp:45-62)
 * and the assembly tasks that implement ScatterReplace_/ScatterAdd_/
 * AddNew*Interactions_ (src/DE/mf2d.cpp:755-901). */
int mfgpu_symbolic_create(int dim, int nx, int ny, int nz, int width, int max_side_length,
                          mfgpu_symbolic** out);
/* The same with task tables for nonsymmetric matrices (every block of every
 * front and separator, both triangles, as the reference's LU-based fronts
 * hold them): the form the separator width 2-3 stencils of the reference
 * fixture need with variable coefficients.  Host only; the GPU factorization
 * stores lower triangles and does not use these tables. */
int mfgpu_symbolic_create_full(int dim, int nx, int ny, int nz, int width, int max_side_length,
                               mfgpu_symbolic** out);
/* The forest schedule of a batch (see mfgpu_batch_create), host only. */
int mfgpu_symbolic_batch_create(int count, const int* dim, const int* nx, const int* ny,
                                const int* nz, const int* width, const int* max_side,
                                mfgpu_symbolic** out);
void mfgpu_symbolic_destroy(mfgpu_symbolic* s);
const char* mfgpu_symbolic_error(void);
/* levels, n_fronts, n_seps, ndof */
int mfgpu_symbolic_sizes(const mfgpu_symbolic* s, int* levels, int* n_fronts, int* n_seps,
                         int64_t* ndof);
/* front f (global id, root first, level by level): level, box, n, m, pointer to
 * its n+m DOFs (pivots then boundary) valid until destroy. */
int mfgpu_symbolic_front(const mfgpu_symbolic* s, int f, int* level, int* box, int* n, int* m,
                         const int** dofs);
/* separator k (global id, level 1 first): level, index in level, size, DOFs,
 * and the two adjacent fronts with the separator's row inside each. */
int mfgpu_symbolic_sep(const mfgpu_symbolic* s, int k, int* level, int* idx, int* size,
                       const int** dofs, int boxes[2], int rows[2]);
/* Assembly tasks.  which = 0: front tasks, 1: separator base tasks, 2:
 * separator accumulation tasks.  Returns the count; `tasks` points at an
 * array of 56-byte records laid out as in the C++ struct mfgpu::Task. */
int64_t mfgpu_symbolic_tasks(const mfgpu_symbolic* s, int which, const void** tasks);
/* Fronts a localized update with these modified DOFs refactors (the leaf-marking
 * rule of src/DE/mf2d.cpp:163-174 followed by root paths): dirty[f] = 1 for
 * each, *flops = their Cholesky-form flops.  Returns the count, -1 on error. */
int64_t mfgpu_symbolic_dirty(const mfgpu_symbolic* s, const int* modified_dofs, int n_modified,
                             unsigned char* dirty, double* flops);
/* Arena layout of front f / separator k: element offset and leading dimension. */
int mfgpu_symbolic_layout(const mfgpu_symbolic* s, int front_or_sep, int id, int64_t* off,
                          int* ld);

#ifdef __cplusplus
}
#endif
#endif /* MFGPU_H */
