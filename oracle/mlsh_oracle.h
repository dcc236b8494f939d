/*
 * CPU restatement of the reference's sparse iterative-solve hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline leg may load it.  The
 * product never links, loads or calls it.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares every
 * routine here with the reference CPU library built from the reference
 * sources (oracle/_ref) and with the committed golden fixtures made from it
 * (tests/golden/make_golden.py).
 *
 * Return codes follow include/monolish/common/monolish_common.hpp:16-21 of
 * the reference: 0 success, -2 maxiter, -3 breakdown, -4 residual NaN.
 */
#ifndef MLSH_ORACLE_H
#define MLSH_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

void oracle_spmv_d(int n, const int *rp, const int *ci, const double *v,
                   const double *x, double *y);
void oracle_spmv_s(int n, const int *rp, const int *ci, const float *v,
                   const float *x, float *y);
/* y = alpha*A*x + beta*y (the alpha/beta overload of blas::matvec). */
void oracle_spmv_ab_d(int n, const int *rp, const int *ci, const double *v,
                      double alpha, const double *x, double beta, double *y);

/* y = A^T x for an n_rows x n_cols CRS A: y zeroed, then rows in order,
 * y[col] += val * x[row] (src/blas/matrix/matvec/crs_matvec.hpp:88-98). */
void oracle_spmv_t_d(int n_rows, int n_cols, const int *rp, const int *ci,
                     const double *v, const double *x, double *y);
void oracle_spmv_t_s(int n_rows, int n_cols, const int *rp, const int *ci,
                     const float *v, const float *x, float *y);

/* COO::sort (src/utils/at_insert_sort/at_insert_sort_coo.cpp:119-145):
 * entries ordered by (row, col); with `merge`, each run of equal (row,
 * col) collapses to one entry holding the run's last value.  Ties keep
 * input order (the reference's quicksort leaves it unspecified).  Returns
 * the entry count after merging; arrays are rewritten in place. */
long oracle_coo_sort_d(long nnz, int *row, int *col, double *val, int merge);
/* CRS::convert(COO) row pointer (src/utils/convert/convert_crs.cpp:9-43)
 * for entries sorted by row. */
void oracle_coo_rowptr(int n_rows, long nnz, const int *row, int *rp);
/* The transpose as CRS: entries of each column in row order. */
void oracle_csr_transpose_d(int n_rows, int n_cols, const int *rp, const int *ci,
                            const double *v, int *rp_t, int *ci_t, double *v_t);

double oracle_dot_d(long n, const double *x, const double *y);
double oracle_nrm2_d(long n, const double *x);
double oracle_dot_s(long n, const float *x, const float *y);

/* precond: 0 none, 1 Jacobi, 2 SOR (relaxation omega), 3 IC(0), 4 ILU(0). */
int oracle_cg_d(int n, const int *rp, const int *ci, const double *v,
                const double *b, double *x, double tol_abs, long maxiter,
                long miniter, int precond, double omega, long *iters,
                double *resid);
int oracle_cg_s(int n, const int *rp, const int *ci, const float *v,
                const float *b, float *x, double tol_abs, long maxiter,
                long miniter, int precond, double omega, long *iters,
                double *resid);
int oracle_bicgstab_d(int n, const int *rp, const int *ci, const double *v,
                      const double *b, double *x, double tol_abs, long maxiter,
                      long miniter, int precond, double omega, long *iters,
                      double *resid);
int oracle_bicgstab_s(int n, const int *rp, const int *ci, const float *v,
                      const float *b, float *x, double tol_abs, long maxiter,
                      long miniter, int precond, double omega, long *iters,
                      double *resid);

/* SOR / IC(0) / ILU(0) (kinds 2 / 3 / 4), rows sorted by column.
 * factor: SOR M = 1/(omega diag) (n values); IC / ILU the factor in A's
 * pattern (nnz values); *pivot = first zero pivot row or -1.  Returns -1
 * for unsorted rows.  apply: z = M^{-1} r. */
int oracle_precond_factor_d(int n, const int *rp, const int *ci, const double *v,
                            int kind, double omega, double *out, long *pivot);
int oracle_precond_factor_s(int n, const int *rp, const int *ci, const float *v,
                            int kind, double omega, float *out, long *pivot);
int oracle_precond_apply_d(int n, const int *rp, const int *ci, const double *v,
                           int kind, double omega, const double *r, double *z);
int oracle_precond_apply_s(int n, const int *rp, const int *ci, const float *v,
                           int kind, double omega, const float *r, float *z);
/* equation::SOR::solve: relative stopping test, history of the relative
 * residual (maxiter entries) if hist is given. */
int oracle_sor_d(int n, const int *rp, const int *ci, const double *v,
                 const double *b, double *x, double omega, double tol,
                 long maxiter, long miniter, double *hist, long *iters,
                 double *resid);
int oracle_sor_s(int n, const int *rp, const int *ci, const float *v,
                 const float *b, float *x, double omega, double tol,
                 long maxiter, long miniter, double *hist, long *iters,
                 double *resid);

/* ||b - A x||_2 / ||b||_2 in double. */
double oracle_true_relres_d(int n, const int *rp, const int *ci,
                            const double *v, const double *b, const double *x);

#ifdef __cplusplus
}
#endif
#endif
