// Cross-translation-unit declarations.  Kernel templates are instantiated in
// exactly one translation unit each; other units call the host launchers
// declared here.
#pragma once
#include "mlsh_internal.cuh"
#include "mlsh_spmv.cuh"
#include "mlsh_vec.cuh"

namespace mlsh {

int init_kernel_attributes();

void build_tiles(const int *rp, int n_rows, std::vector<Tile> &tiles,
                 std::vector<LongRow> &longs, int &n_chunks);

// y_out = alpha*A*x + beta*y_in with the fused dots selected by M0/M1
// (instantiated in mlsh_core.cu for VT = double/float and the mode pairs
// (none,none), (w,none), (w,self), (self,none)).
template <typename VT, int M0, int M1>
cudaError_t launch_spmv_t(const CsrPlan &p, const Handle &h, double alpha,
                          const VT *x, double beta, const VT *y_in, VT *y_out,
                          const VT *w0, const VT *w1, double *dot_out,
                          const int *done, cudaStream_t stream);

// Offset-slot layout of an FP32 plan (mlsh_slots.cu): built when the
// structure qualifies (else p.slots stays null), released with the plan or
// when its values change.  launch_spmv_t uses it whenever it is present.
int slots_build(CsrPlan &p, cudaStream_t s);
void slots_release(CsrPlan &p);
template <int M0, int M1>
cudaError_t launch_spmv_slots(const CsrPlan &p, const Handle &h, double alpha, const float *x,
                              double beta, const float *y_in, float *y_out, const float *w0,
                              const float *w1, double *dot_out, const int *done,
                              cudaStream_t stream);

int plan_diag(const CsrPlan &p, void *out, bool invert, cudaStream_t stream);
int plan_inv_diag(CsrPlan &p, cudaStream_t stream, const void **out);

// Cluster engine (mlsh_cluster.cu).  kind: 0 = CG, 1 = BiCGSTAB, 2 = mixed
// CG (FP32 iteration, FP64 x and true residual; launched with dtype F32,
// records carrying the FP64 values in `aux`).
struct ClusterSystem;
// Rows per CTA for an n-row system (0 if it does not fit 16 CTAs).
int cluster_rows_for(int kind, int dtype, int64_t n, int requested);
// Launches n_clusters clusters of csize CTAs that take systems from
// d_queue (zero it first) until n_systems are done.
int cluster_launch(const Handle &h, int kind, int dtype, bool jac, ClusterSystem *d_systems,
                   int n_systems, unsigned *d_queue, int rpc, int csize, int n_clusters,
                   double budget_s, cudaStream_t stream, double delta = 0.0);
int cluster_max_active(int kind, int dtype, bool jac, int rpc, int csize);
struct ServeRing;
// The serving kernel (FP64, kServeRows rows per CTA) on n_clusters
// clusters of csize CTAs, fed from `ring`.
int cluster_serve_launch(const ServeRing &ring, int csize, int n_clusters, double budget_s,
                         cudaStream_t stream);

// Mixed-precision data kept with an FP64 plan (mlsh_mixed.cu).
void mixed_release(CsrPlan &p);
void mixed_invalidate(CsrPlan &p);

// A^T of an n_rows x n_cols CRS (rows of A^T sorted by column), the entry
// permutation into perm_out if given (mlsh_sort.cu).  Synchronous.
int transpose_build(Handle &h, int n_rows, int n_cols, int nnz, const int *rp, const int *ci,
                    const void *val, int dtype, int *rp_t, int *ci_t, void *val_t,
                    unsigned *perm_out);

// The cached transpose of a plan (mlsh_sort.cu).
void transpose_release(CsrPlan &p);
void transpose_invalidate(CsrPlan &p);

// Mixed-precision BiCGSTAB with reliable updates on the kernel engine
// (mlsh_krylov.cu): p FP64, p32 its FP32 copy (holding A D^-1 when dinv64,
// the FP64 inverse diagonal, is given for Jacobi), r64 an FP64 work vector.
int mixed_bicgstab_kernels(Handle &h, CsrPlan &p, CsrPlan &p32, double *r64,
                           const double *dinv64, const void *b, void *x,
                           const mlsh_solver_opts *opts, double inner_tol,
                           mlsh_solver_result *res);

// Solver-side resources kept on the handle / plan (mlsh_krylov.cu).
void release_solver_graphs(Handle &h);
void release_plan_extras(CsrPlan &p);
void invalidate_plan_extras(CsrPlan &p);

}  // namespace mlsh
