/*
 * CPU restatement of the reference's sparse iterative-solve hot path
 * (TEST INFRASTRUCTURE ONLY -- the checker; see mlsh_oracle.h).
 *
 * Each routine follows the reference step by step:
 *   SpMV        src/blas/matrix/matvec/crs_matvec.hpp:101-108 (OSS row loop:
 *               ytmp = 0; ytmp += val[j] * x[col[j]]; y[i] = ytmp)
 *   alpha/beta  matvec(a,A,x,b,y) overload, src/blas/matrix/matvec/matvec_blas.cpp:3853
 *   dot / nrm2  src/blas/vector/dot.hpp:6-41, nrm2.hpp:6-36 (nrm2 = sqrt(dot(x,x)))
 *   axpy/xpay   src/blas/vector/axpy.hpp:7-34, xpay.hpp:7-36
 *   axpyz       src/blas/vector/axpyz.hpp:7-37
 *   Jacobi      src/equation/jacobi.cpp:12-31 (M = 1/diag(A)), :53-61 (z = M.*r)
 *   none        src/equation/none.cpp:40-46 (z = r)
 *   CG          src/equation/cg.cpp:13-86
 *   BiCGSTAB    src/equation/bicgstab.cpp:13-135
 *
 * The reference computes dot/nrm2 through an external CBLAS (OpenBLAS here),
 * whose summation order is its own; this restatement sums sequentially in
 * double (for float vectors too, rounding the result to float).  The
 * difference is at rounding level and is bounded by the tolerances that
 * tests/test_oracle.py pins against the compiled reference.
 *
 * Built with -ffp-contract=off so that products and sums round separately,
 * as in the reference's x86-64 build (-mavx has no FMA).
 */
#include "mlsh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SOLVER_SUCCESS 0
#define SOLVER_MAXITER (-2)
#define SOLVER_BREAKDOWN (-3)
#define SOLVER_RESIDUAL_NAN (-4)

/* ---------------------------------------------------------------- SpMV --- */
void oracle_spmv_d(int n, const int *rp, const int *ci, const double *v,
                   const double *x, double *y) {
  for (int i = 0; i < n; i++) {
    double t = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];
    y[i] = t;
  }
}

void oracle_spmv_s(int n, const int *rp, const int *ci, const float *v,
                   const float *x, float *y) {
  for (int i = 0; i < n; i++) {
    float t = 0.0f;
    for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];
    y[i] = t;
  }
}

void oracle_spmv_ab_d(int n, const int *rp, const int *ci, const double *v,
                      double alpha, const double *x, double beta, double *y) {
  for (int i = 0; i < n; i++) {
    double t = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];
    y[i] = alpha * t + beta * y[i];
  }
}

/* ------------------------------------------------------ transposed SpMV --- */
void oracle_spmv_t_d(int n_rows, int n_cols, const int *rp, const int *ci,
                     const double *v, const double *x, double *y) {
  for (int j = 0; j < n_cols; j++) y[j] = 0.0;
  for (int i = 0; i < n_rows; i++)
    for (int k = rp[i]; k < rp[i + 1]; k++) y[ci[k]] += v[k] * x[i];
}

void oracle_spmv_t_s(int n_rows, int n_cols, const int *rp, const int *ci,
                     const float *v, const float *x, float *y) {
  for (int j = 0; j < n_cols; j++) y[j] = 0.0f;
  for (int i = 0; i < n_rows; i++)
    for (int k = rp[i]; k < rp[i + 1]; k++) y[ci[k]] += v[k] * x[i];
}

/* ------------------------------------------------------ COO / transpose --- */
typedef struct {
  int row, col;
  long idx;
} coo_key;

static int coo_key_cmp(const void *a, const void *b) {
  const coo_key *p = (const coo_key *)a, *q = (const coo_key *)b;
  if (p->row != q->row) return p->row < q->row ? -1 : 1;
  if (p->col != q->col) return p->col < q->col ? -1 : 1;
  return p->idx < q->idx ? -1 : (p->idx > q->idx ? 1 : 0);
}

long oracle_coo_sort_d(long nnz, int *row, int *col, double *val, int merge) {
  if (nnz <= 0) return 0;
  coo_key *k = (coo_key *)malloc(sizeof(coo_key) * (size_t)nnz);
  double *v = (double *)malloc(sizeof(double) * (size_t)nnz);
  for (long i = 0; i < nnz; i++) {
    k[i].row = row[i];
    k[i].col = col[i];
    k[i].idx = i;
    v[i] = val[i];
  }
  qsort(k, (size_t)nnz, sizeof(coo_key), coo_key_cmp);
  long out = 0;
  for (long i = 0; i < nnz; i++) {
    if (merge && out > 0 && row[out - 1] == k[i].row && col[out - 1] == k[i].col) {
      val[out - 1] = v[k[i].idx]; /* the run keeps its last value */
      continue;
    }
    row[out] = k[i].row;
    col[out] = k[i].col;
    val[out] = v[k[i].idx];
    out++;
  }
  free(k);
  free(v);
  return out;
}

void oracle_coo_rowptr(int n_rows, long nnz, const int *row, int *rp) {
  /* rp[i] = number of entries with row < i */
  long k = 0;
  for (int i = 0; i <= n_rows; i++) {
    while (k < nnz && row[k] < i) k++;
    rp[i] = (int)k;
  }
}

void oracle_csr_transpose_d(int n_rows, int n_cols, const int *rp, const int *ci,
                            const double *v, int *rp_t, int *ci_t, double *v_t) {
  for (int j = 0; j <= n_cols; j++) rp_t[j] = 0;
  for (int k = 0; k < rp[n_rows]; k++) rp_t[ci[k] + 1]++;
  for (int j = 0; j < n_cols; j++) rp_t[j + 1] += rp_t[j];
  int *fill = (int *)malloc(sizeof(int) * (size_t)(n_cols > 0 ? n_cols : 1));
  for (int j = 0; j < n_cols; j++) fill[j] = rp_t[j];
  for (int i = 0; i < n_rows; i++)
    for (int k = rp[i]; k < rp[i + 1]; k++) {
      const int p = fill[ci[k]]++;
      ci_t[p] = i;
      v_t[p] = v[k];
    }
  free(fill);
}

/* ---------------------------------------------------------- reductions --- */
double oracle_dot_d(long n, const double *x, const double *y) {
  double s = 0.0;
  for (long i = 0; i < n; i++) s += x[i] * y[i];
  return s;
}
double oracle_nrm2_d(long n, const double *x) { return sqrt(oracle_dot_d(n, x, x)); }
double oracle_dot_s(long n, const float *x, const float *y) {
  double s = 0.0;
  for (long i = 0; i < n; i++) s += (double)x[i] * (double)y[i];
  return (double)(float)s;
}

double oracle_true_relres_d(int n, const int *rp, const int *ci,
                            const double *v, const double *b, const double *x) {
  double num = 0.0, den = 0.0;
  for (int i = 0; i < n; i++) {
    double t = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];
    double r = b[i] - t;
    num += r * r;
    den += b[i] * b[i];
  }
  return den > 0.0 ? sqrt(num) / sqrt(den) : sqrt(num);
}

/* --------------------------------------------------- generic solvers ----- */
/* The solvers are written once and instantiated for double and float. */
#define DEFINE_SOLVERS(T, SFX, DOT)                                            \
  static void spmv_##SFX(int n, const int *rp, const int *ci, const T *v,      \
                         const T *x, T *y) {                                   \
    for (int i = 0; i < n; i++) {                                              \
      T t = 0;                                                                 \
      for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];            \
      y[i] = t;                                                                \
    }                                                                          \
  }                                                                            \
  /* Jacobi create_precond: M = 1 / diag(A) (crs_getvec.cpp:8-55 diag,       \
     double_arithmetic.cpp:308-330 reciprocal). A missing diagonal is 0. */    \
  static void jacobi_##SFX(int n, const int *rp, const int *ci, const T *v,    \
                           T *M) {                                             \
    for (int i = 0; i < n; i++) {                                              \
      T d = 0;                                                                 \
      for (int j = rp[i]; j < rp[i + 1]; j++)                                  \
        if (ci[j] == i) d = v[j];                                              \
      M[i] = (T)1 / d;                                                         \
    }                                                                          \
  }                                                                            \
  static void apply_##SFX(int n, int precond, const T *M, const T *r, T *z) {  \
    if (precond == 1)                                                          \
      for (int i = 0; i < n; i++) z[i] = M[i] * r[i];                          \
    else                                                                       \
      memcpy(z, r, sizeof(T) * (size_t)n);                                     \
  }                                                                            \
  int oracle_cg_##SFX(int n, const int *rp, const int *ci, const T *v,         \
                      const T *b, T *x, double tol_abs, long maxiter,          \
                      long miniter, int precond, long *iters, double *resid) { \
    T *r = calloc((size_t)n, sizeof(T)), *p = calloc((size_t)n, sizeof(T));    \
    T *q = calloc((size_t)n, sizeof(T)), *z = calloc((size_t)n, sizeof(T));    \
    T *M = calloc((size_t)n, sizeof(T));                                       \
    int ret = SOLVER_MAXITER;                                                  \
    long it_done = maxiter;                                                    \
    if (precond == 1) jacobi_##SFX(n, rp, ci, v, M);                           \
    spmv_##SFX(n, rp, ci, v, x, q); /* cg.cpp:39-40 r = b - Ax */              \
    for (int i = 0; i < n; i++) r[i] = b[i] - q[i];                            \
    apply_##SFX(n, precond, M, r, z); /* cg.cpp:43-44 */                       \
    memcpy(p, z, sizeof(T) * (size_t)n);                                       \
    for (long iter = 0; iter < maxiter; iter++) { /* cg.cpp:46-80 */           \
      spmv_##SFX(n, rp, ci, v, p, q);                                          \
      T tmp = (T)DOT(n, z, r);                                                 \
      T alpha = tmp / (T)DOT(n, p, q);                                         \
      for (int i = 0; i < n; i++) x[i] += alpha * p[i];                        \
      for (int i = 0; i < n; i++) r[i] += -alpha * q[i];                       \
      apply_##SFX(n, precond, M, r, z);                                        \
      T beta = (T)DOT(n, z, r) / tmp;                                          \
      for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];                   \
      T res = (T)sqrt((double)(T)DOT(n, r, r));                                \
      if (res < tol_abs && miniter <= iter + 1) {                              \
        it_done = iter + 1;                                                    \
        ret = SOLVER_SUCCESS;                                                  \
        break;                                                                 \
      }                                                                        \
      if (isnan(res)) {                                                        \
        it_done = iter + 1;                                                    \
        ret = SOLVER_RESIDUAL_NAN;                                             \
        break;                                                                 \
      }                                                                        \
    }                                                                          \
    if (iters) *iters = it_done;                                               \
    if (resid) *resid = (double)(T)sqrt((double)(T)DOT(n, r, r));              \
    free(r); free(p); free(q); free(z); free(M);                               \
    return ret;                                                                \
  }                                                                            \
  int oracle_bicgstab_##SFX(int n, const int *rp, const int *ci, const T *v,   \
                            const T *b, T *x, double tol_abs, long maxiter,    \
                            long miniter, int precond, long *iters,            \
                            double *resid) {                                   \
    size_t sz = sizeof(T) * (size_t)n;                                         \
    T *r = calloc((size_t)n, sizeof(T)), *r0 = calloc((size_t)n, sizeof(T));   \
    T *p = calloc((size_t)n, sizeof(T)), *ph = calloc((size_t)n, sizeof(T));   \
    T *s = calloc((size_t)n, sizeof(T)), *sh = calloc((size_t)n, sizeof(T));   \
    T *vv = calloc((size_t)n, sizeof(T)), *t = calloc((size_t)n, sizeof(T));   \
    T *M = calloc((size_t)n, sizeof(T));                                       \
    T rho_old = 1, rho = 1, alpha = 1, beta, omega = 1;                        \
    int ret = SOLVER_MAXITER;                                                  \
    long it_done = maxiter;                                                    \
    if (precond == 1) jacobi_##SFX(n, rp, ci, v, M);                           \
    spmv_##SFX(n, rp, ci, v, x, r); /* bicgstab.cpp:47-51 */                   \
    for (int i = 0; i < n; i++) r[i] = b[i] - r[i];                            \
    memcpy(r0, r, sz);                                                         \
    for (long iter = 0; iter < maxiter; iter++) { /* bicgstab.cpp:53-130 */    \
      rho = (T)DOT(n, r, r0);                                                  \
      if (rho == 0) {                                                          \
        it_done = iter + 1;                                                    \
        ret = SOLVER_BREAKDOWN;                                                \
        break;                                                                 \
      }                                                                        \
      if (iter == 0) {                                                         \
        memcpy(p, r, sz);                                                      \
      } else {                                                                 \
        beta = (rho / rho_old) * (alpha / omega);                              \
        for (int i = 0; i < n; i++) p[i] += -omega * vv[i];                    \
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];                 \
      }                                                                        \
      apply_##SFX(n, precond, M, p, ph);                                       \
      spmv_##SFX(n, rp, ci, v, ph, vv);                                        \
      alpha = rho / (T)DOT(n, vv, r0);                                         \
      for (int i = 0; i < n; i++) s[i] = -alpha * vv[i] + r[i];                \
      apply_##SFX(n, precond, M, s, sh);                                       \
      spmv_##SFX(n, rp, ci, v, sh, t);                                         \
      omega = (T)DOT(n, t, s) / (T)DOT(n, t, t);                               \
      if (omega == 0) {                                                        \
        it_done = iter + 1;                                                    \
        ret = SOLVER_BREAKDOWN;                                                \
        break;                                                                 \
      }                                                                        \
      for (int i = 0; i < n; i++) x[i] += alpha * ph[i];                       \
      for (int i = 0; i < n; i++) x[i] += omega * sh[i];                       \
      for (int i = 0; i < n; i++) r[i] = -omega * t[i] + s[i];                 \
      T res = (T)sqrt((double)(T)DOT(n, r, r));                                \
      if (res < tol_abs && miniter <= iter + 1) {                              \
        it_done = iter + 1;                                                    \
        ret = SOLVER_SUCCESS;                                                  \
        break;                                                                 \
      }                                                                        \
      if (isnan(res)) {                                                        \
        it_done = iter + 1;                                                    \
        ret = SOLVER_RESIDUAL_NAN;                                             \
        break;                                                                 \
      }                                                                        \
      rho_old = rho;                                                           \
    }                                                                          \
    if (iters) *iters = it_done;                                               \
    if (resid) *resid = (double)(T)sqrt((double)(T)DOT(n, r, r));              \
    free(r); free(r0); free(p); free(ph); free(s); free(sh);                   \
    free(vv); free(t); free(M);                                                \
    return ret;                                                                \
  }

DEFINE_SOLVERS(double, d, oracle_dot_d)
DEFINE_SOLVERS(float, s, oracle_dot_s)
