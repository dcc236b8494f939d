/*
 * mlsh.h -- C ABI of the B200 (sm_100a) sparse iterative-solve library.
 *
 * This is the boundary a host-side binding links against: plain C types,
 * device pointers, sizes, and a CUDA stream passed as `void *`; every call
 * returns an `int` status and never throws, never exits.  The C++ drop-in
 * layer (monolish_b200/cpp, monolish's own class/function names) and the
 * Python test harness both sit on top of these entry points.
 *
 * Each entry point replaces one reference interface; the citation is the
 * reference source it stands in for (paths inside the monolish project).
 *
 * Conventions
 *   dtype        MLSH_F64 (double) or MLSH_F32 (float): the element type of
 *                the matrix values and of every vector in the call.
 *   pointers     device pointers (cudaMalloc'd or equivalent) unless the
 *                name says `host`.  Vectors may be unaligned; 16-byte
 *                aligned vectors take the vectorised path.
 *   streams      `stream` is a cudaStream_t (NULL = legacy default stream).
 *                Calls are asynchronous w.r.t. the host unless stated.
 *   reductions   accumulate in double for both dtypes, in a fixed order:
 *                repeated calls with the same inputs give bit-identical
 *                results.
 *   concurrency  a handle or a plan is used by one stream at a time (they
 *                hold scratch buffers); use one handle per stream.
 */
#ifndef MLSH_H
#define MLSH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ statuses --
 * Solver codes are the reference's (include/monolish/common/
 * monolish_common.hpp:16-21); library errors are new negative codes. */
#define MLSH_SUCCESS 0
#define MLSH_SOLVER_SIZE_ERROR (-1)
#define MLSH_SOLVER_MAXITER (-2)
#define MLSH_SOLVER_BREAKDOWN (-3)
#define MLSH_SOLVER_RESIDUAL_NAN (-4)
#define MLSH_NOT_IMPL (-10)
#define MLSH_ERR_CUDA (-20)         /* a CUDA runtime call failed */
#define MLSH_ERR_INVALID_ARG (-21)  /* NULL handle/pointer, bad dtype, n < 0 */
#define MLSH_ERR_INVALID_CSR (-22)  /* row_ptr not monotone / col out of range */
#define MLSH_ERR_OOM (-23)          /* device allocation failed */
#define MLSH_ERR_TIMEOUT (-24)      /* a bounded device-side wait gave up */
#define MLSH_ERR_NO_DEVICE (-25)    /* no CUDA device / not sm_100 */

#define MLSH_F64 0
#define MLSH_F32 1

#define MLSH_PRECOND_NONE 0   /* equation::none (src/equation/none.cpp:40-46) */
#define MLSH_PRECOND_JACOBI 1 /* equation::Jacobi (src/equation/jacobi.cpp:12-61) */
#define MLSH_PRECOND_SOR 2    /* equation::SOR as preconditioner (src/equation/sor.cpp:12-77) */
#define MLSH_PRECOND_IC 3     /* equation::IC, IC(0) (src/equation/ic.cpp:12-140) */
#define MLSH_PRECOND_ILU 4    /* equation::ILU, ILU(0) (src/equation/ilu.cpp:12-140) */

typedef struct mlsh_handle_s *mlsh_handle;
typedef struct mlsh_csr_plan_s *mlsh_csr_plan;

/* ------------------------------------------------------------- library -- */
/* Version as major*10000 + minor*100 + patch. */
int mlsh_version(void);
/* Human-readable text for a status code (static storage). */
const char *mlsh_status_string(int status);
/* Last CUDA error text recorded by this thread (static per thread). */
const char *mlsh_last_error(void);

/* A handle owns a stream binding and the small scratch buffers used by the
 * reductions and solvers, on the device current at creation.  Replaces the
 * per-call cublasCreate/cusparseCreate of the reference GPU path
 * (src/blas/vector/dot.hpp:21-25, src/blas/matrix/matvec/crs_matvec.hpp:42-64). */
int mlsh_create(mlsh_handle *handle);
int mlsh_destroy(mlsh_handle handle);
int mlsh_set_stream(mlsh_handle handle, void *stream);
int mlsh_get_stream(mlsh_handle handle, void **stream);
int mlsh_synchronize(mlsh_handle handle);

/* ---------------------------------------------------- device memory ----- */
/* Device residency for hosts that include no CUDA headers: these back the
 * send() / recv() / nonfree_recv() / device_free() of vector and CRS
 * (src/utils/system/gpu_comm.cpp:8-183, where the reference maps host
 * arrays with OpenMP target data directives).  Allocations are 256-byte
 * aligned.  The copies are synchronous with respect to the host and ordered
 * on the handle's stream. */
int mlsh_device_alloc(size_t bytes, void **d_ptr);
int mlsh_device_free(void *d_ptr);
int mlsh_memcpy_h2d(mlsh_handle handle, void *d_dst, const void *h_src,
                    size_t bytes);
int mlsh_memcpy_d2h(mlsh_handle handle, void *h_dst, const void *d_src,
                    size_t bytes);
/* The same copies without the host wait, ordered on the handle's stream:
 * they return once the copy is queued.  The host buffer must stay valid and
 * unchanged (h2d) or unread (d2h) until the stream reaches the copy; from
 * page-locked host memory the copy runs asynchronously and can overlap
 * kernels and copies on other streams.  A pipelined form of send()/recv()
 * (gpu_comm.cpp:8-73) for callers that stream inputs in and results out. */
int mlsh_memcpy_h2d_async(mlsh_handle handle, void *d_dst, const void *h_src,
                          size_t bytes);
int mlsh_memcpy_d2h_async(mlsh_handle handle, void *h_dst, const void *d_src,
                          size_t bytes);
/* Device-to-device copy, asynchronous on the handle's stream. */
int mlsh_memcpy_d2d(mlsh_handle handle, void *d_dst, const void *d_src,
                    size_t bytes);

/* --------------------------------------------------------------- CRS ---- */
/* Build an SpMV plan over a device-resident CRS matrix (0-based row_ptr
 * [n_rows+1], col_ind [nnz], val [nnz] of `dtype`), as matrix::CRS<T>
 * holds it (include/monolish/common/monolish_crs.hpp:39-110) once send()
 * has copied it (src/utils/system/gpu_comm.cpp:89-110).  The plan keeps the
 * pointers (it does not copy the arrays; they must outlive it) and derives
 * row tiles from row_ptr: from `host_row_ptr` when given, else from a copy
 * of the device row_ptr.  `validate` != 0 also checks the structure on the
 * host (monotone row_ptr, columns in range) and returns
 * MLSH_ERR_INVALID_CSR on failure.  Synchronous. */
int mlsh_csr_plan_create(mlsh_handle handle, int n_rows, int n_cols, int nnz,
                         const int *d_row_ptr, const int *d_col_ind,
                         const void *d_val, int dtype,
                         const int *host_row_ptr, int validate,
                         mlsh_csr_plan *plan);
int mlsh_csr_plan_destroy(mlsh_csr_plan plan);
/* Values changed in place (same structure): drop cached derived data
 * (inverse diagonal, FP32 copy). */
int mlsh_csr_plan_values_changed(mlsh_csr_plan plan);
/* Introspection for tests and the autotuner: number of row tiles, of long
 * rows split into chunks, and the algorithmic bytes of one SpMV
 * (nnz*(V+4) + (n+1)*4 + 2*n*X). */
int mlsh_csr_plan_info(mlsh_csr_plan plan, int *n_tiles, int *n_long_rows,
                       int64_t *spmv_bytes);

/* SpMV kernel variants (shared-memory pipeline depth x CTAs per SM).  A plan
 * starts with a default; mlsh_csr_plan_autotune times every variant on the
 * plan's own matrix (x: n_cols elements, y: n_rows scratch elements, both
 * of the plan's dtype) and keeps the fastest for all later SpMVs and
 * solves.  Synchronous. */
int mlsh_csr_plan_autotune(mlsh_handle handle, mlsh_csr_plan plan,
                           const void *d_x, void *d_y, int *chosen_variant,
                           double *best_seconds);
int mlsh_csr_plan_set_variant(mlsh_csr_plan plan, int variant);
int mlsh_csr_plan_get_variant(mlsh_csr_plan plan, int *variant,
                              int *n_variants);
/* The short-row limit: rows of up to this many entries (8, 16 or 32) are
 * summed by one thread in row order -- the reference's loop
 * (crs_matvec.hpp:101-108), so those rows of y are bit-identical to it for
 * every limit; longer rows are summed by a warp (within the summation error
 * bound).  mlsh_csr_plan_autotune times the limits that change the work
 * (16 and 32 only when some row is longer than 8, resp. 16) together with
 * the kernel variants and keeps the fastest pair; mlsh_csr_plan_tuning
 * reports the pair in use.  No counterpart in the reference. */
int mlsh_csr_plan_set_short_rows(mlsh_csr_plan plan, int max_len);
int mlsh_csr_plan_tuning(mlsh_csr_plan plan, int *variant, int *short_max);

/* Storage layout of an FP32 plan's SpMV (no counterpart in the reference,
 * whose matvec reads the CRS arrays, crs_matvec.hpp:101-108).
 * MLSH_LAYOUT_CRS: the caller's CRS arrays.  MLSH_LAYOUT_SLOTS: a derived
 * copy in which each slice of 256 rows stores at most 8 column offsets
 * (col - row) once and its values slot by slot, with a one-byte presence
 * mask per row -- stencil matrices on structured grids need no column
 * indices at all.  It applies only when every row is sorted, has no repeated
 * column and at most 8 entries; each row is then summed exactly as the CRS
 * kernel sums it, so y is the same in both layouts.  *applied (optional)
 * reports whether the requested layout is in use.  The mixed-precision
 * solvers pick the slot layout for their FP32 copy by themselves.  The copy
 * is dropped by mlsh_csr_plan_values_changed.  Synchronous. */
#define MLSH_LAYOUT_CRS 0
#define MLSH_LAYOUT_SLOTS 1
int mlsh_csr_plan_set_layout(mlsh_csr_plan plan, int layout, int *applied);
/* The matrix bytes one SpMV reads in the layout in use (values, indices, row
 * pointers or masks): of the plan itself (which = 0), or of the FP32 copy
 * the mixed-precision solvers keep with an FP64 plan (which = 1; *layout =
 * -1 and 0 bytes until a mixed solve has built it).  For roofline
 * accounting. */
int mlsh_csr_plan_storage(mlsh_csr_plan plan, int which, int *layout,
                          int64_t *matrix_bytes);

/* y = alpha*A*x + beta*y.  Replaces blas::matvec(A,x,y) and the
 * matvec(a,A,x,b,y) overload (src/blas/matrix/matvec/matvec_blas.cpp:3849-3877,
 * core src/blas/matrix/matvec/crs_matvec.hpp:8-114).  beta == 0 does not
 * read y.  x and y must not alias. */
int mlsh_spmv(mlsh_handle handle, mlsh_csr_plan plan, double alpha,
              const void *d_x, double beta, void *d_y);

/* d_diag[i] = A(i,i) (0 where the row has no diagonal entry).  Replaces
 * CRS::diag (src/utils/getvec/crs_getvec.cpp:8-55). */
int mlsh_csr_diag(mlsh_handle handle, mlsh_csr_plan plan, void *d_diag);

/* y = alpha*A^T*x + beta*y for the plan's n_rows x n_cols matrix (x has
 * n_rows entries, y n_cols).  Replaces blas::matvec_T(CRS,x,y)
 * (src/blas/matrix/matvec/crs_matvec.hpp:88-98; the reference's OSS path
 * ignores alpha and beta, so parity uses alpha = 1, beta = 0).  The first
 * call builds A^T on the device and keeps it with the plan;
 * mlsh_csr_plan_values_changed refreshes its values. */
int mlsh_spmv_transpose(mlsh_handle handle, mlsh_csr_plan plan, double alpha,
                        const void *d_x, double beta, void *d_y);

/* ------------------------------------------------------ matrix set-up -- */
/* Sorts device COO arrays in place by (row, col), entries with equal
 * (row, col) keeping their input order.  With merge != 0 each such run
 * collapses to one entry holding the run's last value, and *new_nnz is the
 * count left.  Replaces COO::sort(merge)
 * (src/utils/at_insert_sort/at_insert_sort_coo.cpp:119-145), whose
 * quicksort leaves the order of duplicates unspecified.  Indices outside
 * [0,n_rows) x [0,n_cols) give MLSH_ERR_INVALID_ARG. */
int mlsh_coo_sort(mlsh_handle handle, int n_rows, int n_cols, int64_t nnz, int *d_row,
                  int *d_col, void *d_val, int dtype, int merge, int64_t *new_nnz);

/* d_row_ptr[n_rows+1] of the CRS holding a row-sorted COO (its column and
 * value arrays are the CRS's as they are).  Replaces the row-pointer pass of
 * CRS::convert(COO&) (src/utils/convert/convert_crs.cpp:9-43).  Rows out of
 * order or out of range give MLSH_ERR_INVALID_CSR. */
int mlsh_coo_to_csr(mlsh_handle handle, int n_rows, int64_t nnz, const int *d_row,
                    int *d_row_ptr);

/* The transpose of an n_rows x n_cols CRS as an n_cols x n_rows CRS
 * (d_rp_t[n_cols+1], d_ci_t[nnz], d_val_t[nnz]); each of its rows lists
 * the entries of one column of A in row order.  No reference counterpart
 * as a function (the reference transposes inside matvec_T). */
int mlsh_csr_transpose(mlsh_handle handle, int n_rows, int n_cols, int nnz, const int *d_rp,
                       const int *d_ci, const void *d_val, int dtype, int *d_rp_t,
                       int *d_ci_t, void *d_val_t);

/* ------------------------------------------------------ vector BLAS ----- */
/* Results returned to host memory, like blas::dot/nrm2 on the reference GPU
 * path (src/blas/vector/dot.hpp:6-41, nrm2.hpp:6-36); synchronous. */
int mlsh_dot(mlsh_handle handle, int dtype, int64_t n, const void *d_x,
             const void *d_y, double *host_result);
int mlsh_nrm2(mlsh_handle handle, int dtype, int64_t n, const void *d_x,
              double *host_result);
/* Same reductions left on the device (one double at d_result); async. */
int mlsh_dot_device(mlsh_handle handle, int dtype, int64_t n, const void *d_x,
                    const void *d_y, double *d_result);
int mlsh_nrm2_device(mlsh_handle handle, int dtype, int64_t n,
                     const void *d_x, double *d_result);
/* The device dot product above for callers that cannot allocate device
 * memory (a framework that owns the device memory through its own pool, a
 * latency-critical loop that cannot take cudaMalloc's implicit
 * synchronisation): no handle, nothing allocated.  This entry point has no
 * counterpart in the reference.  Same result as mlsh_dot_device.  Its
 * scratch is a static 16,640-byte device array (an arrival counter plus
 * partial sums for at most 2048 CTAs) that every GPU loading the library
 * holds until exit; a device needing more CTAs than that is rejected with
 * MLSH_ERR_INVALID_ARG (see mlsh_last_error).  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress) and should come before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race; order them on one stream.  Runs on `stream` on the current device;
 * asynchronous. */
int mlsh_dot_noalloc(int dtype, int64_t n, const void *d_x, const void *d_y,
                     double *d_result, void *stream);
/* y = alpha*x + y          (src/blas/vector/axpy.hpp:7-34) */
int mlsh_axpy(mlsh_handle handle, int dtype, int64_t n, double alpha,
              const void *d_x, void *d_y);
/* y = x + alpha*y          (src/blas/vector/xpay.hpp:7-36) */
int mlsh_xpay(mlsh_handle handle, int dtype, int64_t n, double alpha,
              const void *d_x, void *d_y);
/* z = alpha*x + y          (src/blas/vector/axpyz.hpp:7-37) */
int mlsh_axpyz(mlsh_handle handle, int dtype, int64_t n, double alpha,
               const void *d_x, const void *d_y, void *d_z);
/* y = x                    (src/blas/vector/copy.hpp:5-16) */
int mlsh_copy(mlsh_handle handle, int dtype, int64_t n, const void *d_x,
              void *d_y);
/* y = a - b                (vml::sub, src/internal/arithmetic/double_arithmetic.cpp:141-168) */
int mlsh_vsub(mlsh_handle handle, int dtype, int64_t n, const void *d_a,
              const void *d_b, void *d_y);
/* y = a .* b               (vml::mul, double_arithmetic.cpp:170-197) */
int mlsh_vmul(mlsh_handle handle, int dtype, int64_t n, const void *d_a,
              const void *d_b, void *d_y);
/* y = 1 ./ a               (vml::reciprocal, double_arithmetic.cpp:308-330) */
int mlsh_vreciprocal(mlsh_handle handle, int dtype, int64_t n,
                     const void *d_a, void *d_y);
/* y[i] = value             (vector(N, value) fill) */
int mlsh_fill(mlsh_handle handle, int dtype, int64_t n, double value,
              void *d_y);

/* ------------------------------------------------------------ solvers --- */
/* Solve engines.
 *   KERNELS  one kernel per step (SpMV+dot, update+dots, direction update),
 *            the loop in a CUDA graph with a device-side while node; any n.
 *   CLUSTER  the whole solve in one launch of one thread-block cluster (up
 *            to 16 CTAs) with the iteration vectors in shared memory and
 *            the gathered vector read across CTAs; for n up to 131,072
 *            (CG, FP64) / 65,536 (BiCGSTAB, FP64), twice that in FP32.  A
 *            wall-clock budget of 60 s per solve ends a solve that does not
 *            terminate with MLSH_ERR_TIMEOUT.
 *   AUTO     CLUSTER when the system fits and maxiter <= 2,000,000, else
 *            KERNELS. */
#define MLSH_ENGINE_AUTO 0
#define MLSH_ENGINE_KERNELS 1
#define MLSH_ENGINE_CLUSTER 2

typedef struct {
  double tol;       /* absolute threshold on ||r||_2, like solver::set_tol
                       (src/equation/cg.cpp:67, equation.cpp:8-11) */
  int64_t maxiter;  /* set_maxiter */
  int64_t miniter;  /* set_miniter */
  int precond;      /* MLSH_PRECOND_NONE / MLSH_PRECOND_JACOBI */
  int use_graph;    /* KERNELS engine: 1: whole solve as one CUDA graph with a
                       device-side while loop (no host round trip); 0: eager
                       launches with a host check every `check_every` steps */
  int check_every;  /* eager mode only; <= 0 picks a default */
  int engine;       /* MLSH_ENGINE_* */
  double *history;     /* optional host buffer: ||r|| after each iteration
                          (solver::set_print_rhistory, cg.cpp:62-65) */
  int64_t history_len; /* capacity of `history` in doubles */
  int cluster_rows;    /* CLUSTER engine: rows per CTA (a power of two >= 1024);
                          0 picks the smallest that fits 16 CTAs */
  int reserved;
  /* Device-side limits on waiting (no counterpart in the reference, which
   * exit()s on a CUDA error, src/internal/monolish_internal.hpp:34-43):
   * a kernel that runs past one gives up, the call returns MLSH_ERR_TIMEOUT
   * and the handle stays usable. */
  double time_limit;   /* wall-clock budget of one solve on the CLUSTER
                          engine (single solves and batches), checked by the
                          kernel at every reduction; <= 0: 60 s */
  int64_t wait_polls;  /* SOR / IC / ILU solves: polls a 32-row block makes for
                          a block it depends on before it gives up; <= 0:
                          2^22 (a few seconds) */
} mlsh_solver_opts;

typedef struct {
  int status;          /* MLSH_SUCCESS / MLSH_SOLVER_MAXITER / ... */
  int outer_iters;     /* mixed-precision solves: refinement steps; else 0 */
  int64_t iters;       /* solver::get_final_iter (mixed: inner iterations) */
  double final_resid;  /* solver::get_final_residual = ||r||_2 (absolute) */
} mlsh_solver_result;

/* Fills `opts` with the reference defaults (tol 1e-8, maxiter SIZE_MAX ->
 * INT64_MAX, miniter 0, Jacobi, graph on). */
int mlsh_solver_opts_default(mlsh_solver_opts *opts);

/* Jacobi-preconditioned (or unpreconditioned) CG on the plan's matrix:
 * x is the initial guess on entry and the solution on exit.  Follows the
 * textbook recurrence of equation::CG (src/equation/cg.cpp:13-86) with the
 * same stopping rule (||r|| < tol && miniter <= iter, NaN check).
 * Synchronous; returns result->status. */
int mlsh_cg_solve(mlsh_handle handle, mlsh_csr_plan plan, const void *d_b,
                  void *d_x, const mlsh_solver_opts *opts,
                  mlsh_solver_result *result);
/* BiCGSTAB, following equation::BiCGSTAB (src/equation/bicgstab.cpp:13-135),
 * including its breakdown checks (rho == 0, omega == 0). */
int mlsh_bicgstab_solve(mlsh_handle handle, mlsh_csr_plan plan,
                        const void *d_b, void *d_x,
                        const mlsh_solver_opts *opts,
                        mlsh_solver_result *result);

/* Mixed precision (no reference counterpart; the reference solves in the
 * matrix's own precision): FP32 inner CG / BiCGSTAB iterations on an FP32
 * copy of an FP64 plan's values (with 16-bit column offsets when every row
 * tile's columns span < 65,536), inside an FP64 iterative-refinement loop
 * that computes the true residual r = b - A x and the update x += d in
 * FP64.  opts->tol is the absolute threshold on that true residual;
 * inner_tol (0 < inner_tol < 1) is the inner solves' relative tolerance;
 * opts->maxiter bounds the total inner iterations.  result->iters counts
 * inner iterations, result->outer_iters the refinement steps, and
 * opts->history (if given) receives the true residual per outer step.
 * The FP32 copy is derived on the first call and kept with the plan until
 * its values change (mlsh_csr_plan_values_changed). */
int mlsh_cg_solve_mixed(mlsh_handle handle, mlsh_csr_plan plan, const void *d_b,
                        void *d_x, const mlsh_solver_opts *opts, double inner_tol,
                        mlsh_solver_result *result);
int mlsh_bicgstab_solve_mixed(mlsh_handle handle, mlsh_csr_plan plan,
                              const void *d_b, void *d_x,
                              const mlsh_solver_opts *opts, double inner_tol,
                              mlsh_solver_result *result);

/* ------------------------------------------ SOR / IC / ILU (factored) -- */
/* Preconditioners that need triangular sweeps (the reference's SOR, IC and
 * ILU; its IC and ILU run only on the GPU, through cuSPARSE csric02 /
 * csrilu02 and csrsv2).  All work -- the factorization and every sweep --
 * runs in this library's kernels.  Rows must be sorted by column
 * (MLSH_ERR_INVALID_CSR otherwise); the matrix must be square.
 *
 *   MLSH_PRECOND_SOR  M = 1 / (omega * diag(A)); apply z = M^{-1} r is a
 *                     forward sweep y_i = (r_i - sum_{j<i} a_ij y_j) M_i then
 *                     a backward sweep z_i = y_i - (sum_{j>i} a_ij z_j) M_i
 *                     (src/equation/kernel/sor_kernel.hpp:42-72).  The
 *                     sweeps read the plan's values at apply time.
 *   MLSH_PRECOND_IC   IC(0): L with A ~ L L^T on A's lower pattern; apply
 *                     solves L y = r, L^T z = y.
 *   MLSH_PRECOND_ILU  ILU(0): A ~ L U on A's pattern, L unit lower; apply
 *                     solves L y = r, U z = y.
 * The object refers to the plan, which must outlive it; after the plan's
 * values change, create it again (the reference builds it in every solve).
 * Apply and the solves below run on the handle's stream; one object is used
 * by one stream at a time. */
typedef struct mlsh_precond_s *mlsh_precond;

/* omega: SOR relaxation (solver::set_omega, default 1.9); ignored for IC /
 * ILU.  Synchronous. */
int mlsh_precond_create(mlsh_handle handle, mlsh_csr_plan plan, int kind,
                        double omega, mlsh_precond *out);
/* First zero pivot of an IC / ILU factorization, like
 * cusparseXcsric02_zeroPivot / cusparseXcsrilu02_zeroPivot in
 * src/equation/kernel/{ic,ilu}_kernel.hpp: *row = the first row without a
 * stored diagonal (*structural = 1) or whose pivot is zero (ILU: u_ii == 0;
 * IC: a_ii - sum l_ik^2 <= 0), -1 if there is none.  SOR: always -1. */
int mlsh_precond_zero_pivot(mlsh_precond pc, int64_t *row, int *structural);
/* z = M^{-1} r (equation::SOR/IC/ILU::apply_precond); r and z distinct. */
int mlsh_precond_apply(mlsh_handle handle, mlsh_precond pc, const void *d_r,
                       void *d_z);
/* Copies the factor: IC / ILU its values in the plan's pattern (nnz
 * elements; IC fills the lower triangle with L and keeps A's upper
 * triangle), SOR the vector M (n elements). */
int mlsh_precond_factor(mlsh_handle handle, mlsh_precond pc, void *d_out);
int mlsh_precond_destroy(mlsh_precond pc);
/* The sweeps' schedules: the length of the longest dependency chain of
 * 32-row blocks in the lower (forward) and upper (backward) sweep -- each
 * link is one wait for another warp's result, so an apply takes at least
 * (levels_lower + levels_upper) such hops -- and the block count. */
int mlsh_precond_info(mlsh_precond pc, int *levels_lower, int *levels_upper,
                      int64_t *blocks);
/* Which kernel runs each sweep: MLSH_SWEEP_FLAGS (blocks spread over the
 * GPU, one warp per block, per-block flags between warps), MLSH_SWEEP_CTA
 * (one CTA, the solution in shared memory, a barrier between levels) or
 * MLSH_SWEEP_RING (one CTA as before, each block's matrix-only row state
 * precomputed at creation and streamed into a shared-memory ring by bulk
 * copies ahead of the level being solved).  -1: the sweep does not exist
 * (SOR as a solver has no upper sweep). */
#define MLSH_SWEEP_FLAGS 0
#define MLSH_SWEEP_CTA 1
#define MLSH_SWEEP_RING 2
int mlsh_precond_sweep_form(mlsh_precond pc, int *lower, int *upper);

/* CG / BiCGSTAB preconditioned by `pc` (the reference's solvers with
 * set_create_precond / set_apply_precond bound to equation::SOR, IC or
 * ILU): the same recurrences, stopping rule and codes as mlsh_cg_solve /
 * mlsh_bicgstab_solve, with z = M^{-1} r from the sweeps.  opts->precond
 * and opts->engine are ignored (kernel engine). */
int mlsh_cg_solve_precond(mlsh_handle handle, mlsh_csr_plan plan, mlsh_precond pc,
                          const void *d_b, void *d_x, const mlsh_solver_opts *opts,
                          mlsh_solver_result *result);
int mlsh_bicgstab_solve_precond(mlsh_handle handle, mlsh_csr_plan plan,
                                mlsh_precond pc, const void *d_b, void *d_x,
                                const mlsh_solver_opts *opts,
                                mlsh_solver_result *result);
/* The SOR iteration of equation::SOR::solve (src/equation/sor.cpp:92-162):
 * x += (D/omega + L)^{-1} (b - A x) until ||b - A x|| / ||b|| < opts->tol
 * (relative, as the reference's SOR checks it) and miniter <= iter.
 * result->final_resid is the absolute ||b - A x|| of the last check, the
 * history (if requested) the relative one.  opts->precond must be
 * MLSH_PRECOND_NONE (the solver's own preconditioner). */
int mlsh_sor_solve(mlsh_handle handle, mlsh_csr_plan plan, const void *d_b,
                   void *d_x, double omega, const mlsh_solver_opts *opts,
                   mlsh_solver_result *result);

/* ------------------------------------------------------ batched solves -- */
/* Thousands of independent, uneven systems solved together (no reference
 * counterpart: the reference solves one system per solve() call).
 *
 * Storage: the systems' CRS matrices concatenated.  System k owns rows
 * [row_off[k], row_off[k+1]) of the concatenated vectors; `d_row_ptr`
 * (total_rows + 1 entries) holds offsets into the concatenated col/val
 * arrays, and column indices are local to their system (0 .. n_k - 1).
 * Every system must fit the cluster engine (n_k <= 131,072 CG / 65,536
 * BiCGSTAB in FP64).
 *
 * mlsh_batch_create groups the systems by the cluster size they need
 * (largest first).  mlsh_batch_solve launches one persistent cluster
 * kernel per group on its own stream; each cluster takes systems from the
 * group's queue and solves them start to finish, so systems converge (and
 * retire) independently and freed SMs go to the next group. */
typedef struct mlsh_batch_s *mlsh_batch;

int mlsh_batch_create(mlsh_handle handle, int n_systems, const int64_t *host_row_off,
                      const int *d_row_ptr, const int *d_col_ind, const void *d_val,
                      int dtype, mlsh_batch *batch);
int mlsh_batch_destroy(mlsh_batch batch);
/* kind 0 = CG, 1 = BiCGSTAB.  d_b / d_x: concatenated right-hand sides and
 * initial guesses (solutions on exit).  host_tol: per-system absolute
 * tolerances (NULL: opts->tol for all).  opts: maxiter, miniter, precond.
 * host_status / host_iters / host_resid (may be NULL): per-system results
 * in input order.  Synchronous; returns MLSH_SUCCESS when every system
 * converged, else the first non-success status. */
int mlsh_batch_solve(mlsh_handle handle, mlsh_batch batch, int kind, const void *d_b,
                     void *d_x, const double *host_tol, const mlsh_solver_opts *opts,
                     int *host_status, int64_t *host_iters, double *host_resid);

/* Autotuner of the batch's bins and cluster shapes (no reference
 * counterpart).  Each system is solved by a cluster of CTAs holding slices
 * of its rows: the widest slice (rows per CTA, a power of two) under a cap
 * that fits the engine, which sets both how many CTAs the system takes and
 * the group -- one persistent launch -- it joins.  This times one full
 * batched solve of `kind` (0 CG, 1 BiCGSTAB, 2 mixed-precision CG with
 * inner_tol as in mlsh_batch_cg_solve_mixed; inner_tol is ignored for 0
 * and 1) for every cap from 1,024 to 16,384 rows that changes the grouping,
 * keeps the fastest for later solves of that kind, and restores d_x (the
 * initial guess) afterwards.  Allocates one copy of x; synchronous. */
int mlsh_batch_autotune(mlsh_handle handle, mlsh_batch batch, int kind, const void *d_b,
                        void *d_x, const double *host_tol, const mlsh_solver_opts *opts,
                        double inner_tol, int *chosen_cap, double *best_seconds);
/* The rows-per-CTA cap in use for `kind` (0 CG, 1 BiCGSTAB, 2 mixed CG) and
 * the number of groups (bins) it makes. */
int mlsh_batch_info(mlsh_batch batch, int kind, int *rows_per_cta_cap, int *n_groups);

/* The batch's Jacobi-CG solves in mixed precision (no reference
 * counterpart): FP32 matrix values and FP32 iteration vectors inside each
 * cluster, the solution and the true residual in FP64.  The FP64 solution
 * and residual are refreshed whenever the iterated residual has fallen by
 * inner_tol since the last refresh (reliable updates); the stopping test
 * (host_tol / opts->tol, absolute) is on the true residual.  The batch must
 * hold FP64 values; its FP32 copy is made on the first call.  host_iters
 * receives FP32 iterations, host_resid the final true ||b - A x||. */
int mlsh_batch_cg_solve_mixed(mlsh_handle handle, mlsh_batch batch, const void *d_b,
                              void *d_x, const double *host_tol,
                              const mlsh_solver_opts *opts, double inner_tol,
                              int *host_status, int64_t *host_iters, double *host_resid);

/* ------------------------------------------------------------- serving -- */
/* A solve server (no reference counterpart): requests of different sizes
 * are submitted from any host thread while others run; a scheduler thread
 * admits them in arrival order while their device-memory footprint fits
 * the budget, uploads them, and runs them concurrently:
 *   - plain-FP64 requests that fit a 16-CTA cluster (n <= 65,536) go to
 *     persistent cluster kernels that claim work from a ring the host
 *     publishes into while they run (continuous batching: a finished
 *     cluster retires its system and takes the next one mid-flight);
 *   - larger or mixed-precision requests run on worker lanes (one handle
 *     and stream each), overlapping with the cluster kernels and each other.
 * A request's host arrays (row_ptr, col_ind, val, b, x0) must stay valid
 * until the request completes; x_out receives the solution. */
#define MLSH_PENDING 1 /* mlsh_server_poll: not finished yet */

typedef struct mlsh_server_s *mlsh_server;

typedef struct {
  int kind;            /* 0 CG, 1 BiCGSTAB */
  int precision;       /* 0 plain FP64, 1 mixed FP32/FP64 */
  int precond;         /* MLSH_PRECOND_* */
  int n;               /* rows = columns */
  int nnz;
  int reserved;
  const int *row_ptr;  /* host CRS (0-based) */
  const int *col_ind;
  const double *val;
  const double *b;     /* host right-hand side */
  const double *x0;    /* host initial guess, or NULL for zeros */
  double *x_out;       /* host buffer for the solution, or NULL */
  double tol;          /* absolute ||r|| threshold */
  int64_t maxiter;
  double inner_tol;    /* mixed precision: inner relative tolerance */
} mlsh_request;

typedef struct {
  int status;
  int path;            /* 0 cluster ring, 1 worker lane */
  int64_t iters;
  double resid;
  double t_submit;     /* seconds on the server's steady clock */
  double t_admit;
  double t_done;
} mlsh_request_result;

/* memory_budget_bytes: device bytes the admitted requests may hold;
 * n_lanes: worker lanes for large / mixed requests (>= 1). */
int mlsh_server_create(size_t memory_budget_bytes, int n_lanes, mlsh_server *server);
int mlsh_server_submit(mlsh_server server, const mlsh_request *request,
                       int64_t *request_id);
/* poll: MLSH_SUCCESS and the result when done, MLSH_PENDING otherwise;
 * wait blocks until done.  A returned result releases the request id (a
 * later poll or wait on it is MLSH_ERR_INVALID_ARG). */
int mlsh_server_poll(mlsh_server server, int64_t request_id, mlsh_request_result *result);
int mlsh_server_wait(mlsh_server server, int64_t request_id, mlsh_request_result *result);
/* Blocks until every submitted request has completed. */
int mlsh_server_drain(mlsh_server server);
/* Seconds on the server's steady clock (the clock of the result times). */
double mlsh_server_now(mlsh_server server);
/* Counters since creation: serving-kernel launches (each runs until its
 * ring stays empty for a short idle period) and requests solved on lanes. */
int mlsh_server_stats(mlsh_server server, int64_t *ring_launches, int64_t *lane_solves);
int mlsh_server_destroy(mlsh_server server);

#ifdef __cplusplus
}
#endif
#endif /* MLSH_H */
