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

/* ------------------------------------------- SOR / IC(0) / ILU(0) ------ */
/* Kinds as in the library: 2 SOR, 3 IC, 4 ILU.
 *   SOR  src/equation/sor.cpp:29-32 (M = 1/(omega diag)), the sweeps of
 *        src/equation/kernel/sor_kernel.hpp:42-72 (precond) and 6-23
 *        (the solver's lower sweep), the solver loop sor.cpp:92-162.
 *   IC / ILU  the reference runs cuSPARSE csric02 / csrilu02 (zero fill-in
 *        incomplete Cholesky / LU on A's pattern) and two csrsv2 solves;
 *        restated here as the row-by-row algorithms: ILU(0) in IKJ form
 *        (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed.,
 *        Alg. 10.4), IC(0) as the row-oriented Cholesky recurrence on the
 *        lower triangle.  Rows must be sorted by column. */
#define PC_SOR 2
#define PC_IC 3
#define PC_ILU 4

/* lo[i] = first entry of row i with col >= i, up[i] = first with col > i.
 * Returns -1 if a row is not sorted, else the first row without a stored
 * diagonal (n if every row has one). */
static long split_rows_c(int n, const int *rp, const int *ci, int *lo, int *up) {
  long missing = n;
  for (int i = 0; i < n; i++) {
    const int b = rp[i], e = rp[i + 1];
    int l = e, u = e;
    for (int j = b; j < e; j++) {
      if (j > b && ci[j] <= ci[j - 1]) return -1;
      if (l == e && ci[j] >= i) l = j;
      if (u == e && ci[j] > i) u = j;
    }
    lo[i] = l;
    up[i] = u;
    if (u == l && missing == n) missing = i;
  }
  return missing;
}

/* Position of column c in the sorted range ci[lo, hi), -1 if absent. */
static int find_col(const int *ci, int lo, int hi, int c) {
  int a = lo, b = hi;
  while (a < b) {
    const int mid = a + (b - a) / 2;
    if (ci[mid] < c) a = mid + 1;
    else b = mid;
  }
  return (a < hi && ci[a] == c) ? a : -1;
}

#define DEFINE_SWEEPS(T, SFX, SQRT)                                            \
  static void transpose_##SFX(int n, const int *rp, const int *ci, const T *v, \
                              int *rpt, int *cit, T *vt) {                     \
    int *fill = calloc((size_t)n + 1, sizeof(int));                            \
    memset(rpt, 0, sizeof(int) * ((size_t)n + 1));                             \
    for (int j = 0; j < rp[n]; j++) rpt[ci[j] + 1]++;                          \
    for (int i = 0; i < n; i++) rpt[i + 1] += rpt[i];                          \
    for (int i = 0; i < n; i++)                                                \
      for (int j = rp[i]; j < rp[i + 1]; j++) {                                \
        const int q = rpt[ci[j]] + fill[ci[j]]++;                              \
        cit[q] = i;                                                            \
        vt[q] = v[j];                                                          \
      }                                                                        \
    free(fill);                                                                \
  }                                                                            \
  /* forward: y_i = (r_i - sum_{j<i} a_ij y_j) then * M_i (SOR), as is       \
     (ILU, unit L) or / l_ii (IC); ascending j (sor_kernel.hpp:50-58). */      \
  static void fwd_##SFX(int kind, int n, const int *rp, const int *ci,         \
                        const T *a, const int *lo, const int *up, const T *M,  \
                        const T *r, T *y) {                                    \
    for (int i = 0; i < n; i++) {                                              \
      T acc = r[i];                                                            \
      for (int j = rp[i]; j < lo[i]; j++) acc = acc - a[j] * y[ci[j]];         \
      if (kind == PC_SOR) y[i] = acc * M[i];                                   \
      else if (kind == PC_ILU) y[i] = acc;                                     \
      else y[i] = acc / (up[i] > lo[i] ? a[lo[i]] : (T)0);                     \
    }                                                                          \
  }                                                                            \
  /* backward.  SOR (sor_kernel.hpp:59-68): tmp is a double ("auto tmp =    \
     0.0"), z_i = y_i - tmp * M_i.  IC / ILU: z_i = (y_i - sum_{j>i} u_ij    \
     z_j) / u_ii, ascending j. */                                              \
  static void bwd_##SFX(int kind, int n, const int *rp, const int *ci,         \
                        const T *a, const int *lo, const int *up, const T *M,  \
                        const T *y, T *z) {                                    \
    for (int i = n - 1; i >= 0; i--) {                                         \
      if (kind == PC_SOR) {                                                    \
        double tmp = 0.0;                                                      \
        for (int j = up[i]; j < rp[i + 1]; j++) tmp += a[j] * z[ci[j]];        \
        z[i] = (T)((double)y[i] - tmp * (double)M[i]);                         \
      } else {                                                                 \
        T acc = y[i];                                                          \
        for (int j = up[i]; j < rp[i + 1]; j++) acc = acc - a[j] * z[ci[j]];   \
        z[i] = acc / (up[i] > lo[i] ? a[lo[i]] : (T)0);                        \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* ILU(0): for each stored k < i ascending, a_ik /= a_kk, then            \
     a_ij -= a_ik a_kj for stored j > k with a_kj stored.  Returns the     \
     first row whose pivot u_ii is zero (or missing), -1 if none. */          \
  static long ilu0_##SFX(int n, const int *rp, const int *ci, const int *lo,   \
                         const int *up, T *f) {                                \
    long piv = -1;                                                             \
    for (int i = 0; i < n; i++) {                                              \
      for (int q = rp[i]; q < lo[i]; q++) {                                    \
        const int k = ci[q];                                                   \
        const T ukk = up[k] > lo[k] ? f[lo[k]] : (T)0;                         \
        const T l = f[q] / ukk;                                                \
        f[q] = l;                                                              \
        for (int p = q + 1; p < rp[i + 1]; p++) {                              \
          const int pos = find_col(ci, up[k], rp[k + 1], ci[p]);               \
          if (pos >= 0) f[p] = f[p] - l * f[pos];                              \
        }                                                                      \
      }                                                                        \
      if (piv < 0 && (!(up[i] > lo[i]) || f[lo[i]] == (T)0)) piv = i;          \
    }                                                                          \
    return piv;                                                                \
  }                                                                            \
  /* IC(0) on the lower triangle: l_ik = (a_ik - sum_{m<k} l_im l_km) /     \
     l_kk, l_ii = sqrt(a_ii - sum_{m<i} l_im^2), sums ascending in m over    \
     stored positions.  Returns the first row with a_ii - sum <= 0. */        \
  static long ic0_##SFX(int n, const int *rp, const int *ci, const int *lo,    \
                        const int *up, T *f) {                                 \
    long piv = -1;                                                             \
    for (int i = 0; i < n; i++) {                                              \
      for (int q = rp[i]; q < lo[i]; q++) {                                    \
        const int k = ci[q];                                                   \
        T s = f[q];                                                            \
        for (int p = rp[i]; p < q; p++) {                                      \
          const int pos = find_col(ci, rp[k], lo[k], ci[p]);                   \
          if (pos >= 0) s = s - f[p] * f[pos];                                 \
        }                                                                      \
        f[q] = s / (up[k] > lo[k] ? f[lo[k]] : (T)0);                          \
      }                                                                        \
      const int has = up[i] > lo[i];                                           \
      T d = has ? f[lo[i]] : (T)0;                                             \
      for (int p = rp[i]; p < lo[i]; p++) d = d - f[p] * f[p];                 \
      if (piv < 0 && !(d > (T)0)) piv = i;                                     \
      if (has) f[lo[i]] = SQRT(d);                                             \
    }                                                                          \
    return piv;                                                                \
  }                                                                            \
  /* Builds a kind's data; solver_scale: the SOR solver's omega/diag.      \
     Returns -1 for unsorted rows. */                                          \
  static int factor_build_##SFX(int kind, double omega, int solver_scale,      \
                                int n, const int *rp, const int *ci,           \
                                const T *v, T **M, T **f, int **lo, int **up,  \
                                int **rpt, int **cit, T **ft, int **lot,       \
                                int **upt, long *piv) {                        \
    *lo = calloc((size_t)n + 1, sizeof(int));                                  \
    *up = calloc((size_t)n + 1, sizeof(int));                                  \
    const long miss = split_rows_c(n, rp, ci, *lo, *up);                       \
    *piv = -1;                                                                 \
    if (miss < 0) return -1;                                                   \
    if (kind == PC_SOR) {                                                      \
      const T w = solver_scale ? (T)(1.0 / (double)(T)omega) : (T)omega;       \
      if (!*M) *M = calloc((size_t)n + 1, sizeof(T));                          \
      for (int i = 0; i < n; i++) {                                            \
        const T d = (*up)[i] > (*lo)[i] ? v[(*lo)[i]] : (T)0;                  \
        (*M)[i] = (T)1 / (w * d);                                              \
      }                                                                        \
      return 0;                                                                \
    }                                                                          \
    const int nnz = rp[n];                                                     \
    *f = calloc((size_t)nnz + 1, sizeof(T));                                   \
    memcpy(*f, v, sizeof(T) * (size_t)nnz);                                    \
    if (miss < n) *piv = miss;                                                 \
    const long p2 = kind == PC_IC ? ic0_##SFX(n, rp, ci, *lo, *up, *f)         \
                                  : ilu0_##SFX(n, rp, ci, *lo, *up, *f);       \
    if (*piv < 0) *piv = p2;                                                   \
    if (kind == PC_IC) {                                                       \
      *rpt = calloc((size_t)n + 1, sizeof(int));                               \
      *cit = calloc((size_t)nnz + 1, sizeof(int));                             \
      *ft = calloc((size_t)nnz + 1, sizeof(T));                                \
      *lot = calloc((size_t)n + 1, sizeof(int));                               \
      *upt = calloc((size_t)n + 1, sizeof(int));                               \
      transpose_##SFX(n, rp, ci, *f, *rpt, *cit, *ft);                         \
      split_rows_c(n, *rpt, *cit, *lot, *upt);                                 \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
  static void sweep_apply_##SFX(int kind, int n, const int *rp, const int *ci, \
                                const T *v, const T *f, const T *M,            \
                                const int *lo, const int *up, const int *rpt,  \
                                const int *cit, const T *ft, const int *lot,   \
                                const int *upt, T *y, const T *r, T *z) {      \
    if (kind == PC_SOR) {                                                      \
      fwd_##SFX(PC_SOR, n, rp, ci, v, lo, up, M, r, y);                        \
      bwd_##SFX(PC_SOR, n, rp, ci, v, lo, up, M, y, z);                        \
    } else if (kind == PC_ILU) {                                               \
      fwd_##SFX(PC_ILU, n, rp, ci, f, lo, up, M, r, y);                        \
      bwd_##SFX(PC_ILU, n, rp, ci, f, lo, up, M, y, z);                        \
    } else {                                                                   \
      fwd_##SFX(PC_IC, n, rp, ci, f, lo, up, M, r, y);                         \
      bwd_##SFX(PC_IC, n, rpt, cit, ft, lot, upt, M, y, z);                    \
    }                                                                          \
  }

DEFINE_SWEEPS(double, d, sqrt)
DEFINE_SWEEPS(float, s, sqrtf)

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
  /* The preconditioner of a solve: none, Jacobi (M), or a sweep kind     \
     (SOR / IC / ILU, see oracle_precond_*). */                              \
  typedef struct {                                                             \
    int kind, n;                                                               \
    const int *rp, *ci;                                                        \
    const T *v;                                                                \
    T *M, *f, *ft, *y;                                                         \
    int *lo, *up, *rpt, *cit, *lot, *upt;                                      \
  } pc_##SFX;                                                                  \
  static void apply_##SFX(const pc_##SFX *pc, const T *r, T *z) {              \
    const int n = pc->n;                                                       \
    if (pc->kind == 1)                                                         \
      for (int i = 0; i < n; i++) z[i] = pc->M[i] * r[i];                      \
    else if (pc->kind >= 2)                                                    \
      sweep_apply_##SFX(pc->kind, n, pc->rp, pc->ci, pc->v, pc->f, pc->M,      \
                        pc->lo, pc->up, pc->rpt, pc->cit, pc->ft, pc->lot,     \
                        pc->upt, pc->y, r, z);                                 \
    else                                                                       \
      memcpy(z, r, sizeof(T) * (size_t)n);                                     \
  }                                                                            \
  static void pc_free_##SFX(pc_##SFX *pc) {                                    \
    free(pc->M); free(pc->f); free(pc->ft); free(pc->y); free(pc->lo);        \
    free(pc->up); free(pc->rpt); free(pc->cit); free(pc->lot); free(pc->upt); \
  }                                                                            \
  static void pc_init_##SFX(pc_##SFX *pc, int kind, double omega, int n,       \
                            const int *rp, const int *ci, const T *v) {        \
    memset(pc, 0, sizeof(*pc));                                                \
    pc->kind = kind; pc->n = n; pc->rp = rp; pc->ci = ci; pc->v = v;           \
    pc->M = calloc((size_t)n + 1, sizeof(T));                                  \
    if (kind == 1) jacobi_##SFX(n, rp, ci, v, pc->M);                          \
    if (kind >= 2) {                                                           \
      long piv;                                                                \
      factor_build_##SFX(kind, omega, 0, n, rp, ci, v, &pc->M, &pc->f,         \
                         &pc->lo, &pc->up, &pc->rpt, &pc->cit, &pc->ft,        \
                         &pc->lot, &pc->upt, &piv);                            \
      pc->y = calloc((size_t)n + 1, sizeof(T));                                \
    }                                                                          \
  }                                                                            \
  int oracle_cg_##SFX(int n, const int *rp, const int *ci, const T *v,         \
                      const T *b, T *x, double tol_abs, long maxiter,          \
                      long miniter, int precond, double omega, long *iters,    \
                      double *resid) {                                         \
    T *r = calloc((size_t)n, sizeof(T)), *p = calloc((size_t)n, sizeof(T));    \
    T *q = calloc((size_t)n, sizeof(T)), *z = calloc((size_t)n, sizeof(T));    \
    pc_##SFX pc;                                                               \
    int ret = SOLVER_MAXITER;                                                  \
    long it_done = maxiter;                                                    \
    pc_init_##SFX(&pc, precond, omega, n, rp, ci, v);                          \
    spmv_##SFX(n, rp, ci, v, x, q); /* cg.cpp:39-40 r = b - Ax */              \
    for (int i = 0; i < n; i++) r[i] = b[i] - q[i];                            \
    apply_##SFX(&pc, r, z); /* cg.cpp:43-44 */                                 \
    memcpy(p, z, sizeof(T) * (size_t)n);                                       \
    for (long iter = 0; iter < maxiter; iter++) { /* cg.cpp:46-80 */           \
      spmv_##SFX(n, rp, ci, v, p, q);                                          \
      T tmp = (T)DOT(n, z, r);                                                 \
      T alpha = tmp / (T)DOT(n, p, q);                                         \
      for (int i = 0; i < n; i++) x[i] += alpha * p[i];                        \
      for (int i = 0; i < n; i++) r[i] += -alpha * q[i];                       \
      apply_##SFX(&pc, r, z);                                                  \
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
    free(r); free(p); free(q); free(z); pc_free_##SFX(&pc);                    \
    return ret;                                                                \
  }                                                                            \
  int oracle_bicgstab_##SFX(int n, const int *rp, const int *ci, const T *v,   \
                            const T *b, T *x, double tol_abs, long maxiter,    \
                            long miniter, int precond, double omega_pc,        \
                            long *iters, double *resid) {                      \
    size_t sz = sizeof(T) * (size_t)n;                                         \
    T *r = calloc((size_t)n, sizeof(T)), *r0 = calloc((size_t)n, sizeof(T));   \
    T *p = calloc((size_t)n, sizeof(T)), *ph = calloc((size_t)n, sizeof(T));   \
    T *s = calloc((size_t)n, sizeof(T)), *sh = calloc((size_t)n, sizeof(T));   \
    T *vv = calloc((size_t)n, sizeof(T)), *t = calloc((size_t)n, sizeof(T));   \
    pc_##SFX pc;                                                               \
    T rho_old = 1, rho = 1, alpha = 1, beta, omega = 1;                        \
    int ret = SOLVER_MAXITER;                                                  \
    long it_done = maxiter;                                                    \
    pc_init_##SFX(&pc, precond, omega_pc, n, rp, ci, v);                       \
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
      apply_##SFX(&pc, p, ph);                                                 \
      spmv_##SFX(n, rp, ci, v, ph, vv);                                        \
      alpha = rho / (T)DOT(n, vv, r0);                                         \
      for (int i = 0; i < n; i++) s[i] = -alpha * vv[i] + r[i];                \
      apply_##SFX(&pc, s, sh);                                                 \
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
    free(vv); free(t); pc_free_##SFX(&pc);                                     \
    return ret;                                                                \
  }

DEFINE_SOLVERS(double, d, oracle_dot_d)
DEFINE_SOLVERS(float, s, oracle_dot_s)

/* ---------------------------------------- SOR / IC / ILU entry points ---- */
#define DEFINE_PC_EXPORTS(T, SFX, DOT)                                         \
  int oracle_precond_factor_##SFX(int n, const int *rp, const int *ci,         \
                                  const T *v, int kind, double omega, T *out,  \
                                  long *pivot) {                               \
    T *M = NULL, *f = NULL, *ft = NULL;                                        \
    int *lo = NULL, *up = NULL, *rpt = NULL, *cit = NULL, *lot = NULL,         \
        *upt = NULL;                                                           \
    long piv = -1;                                                             \
    const int st = factor_build_##SFX(kind, omega, 0, n, rp, ci, v, &M, &f,    \
                                      &lo, &up, &rpt, &cit, &ft, &lot, &upt,   \
                                      &piv);                                   \
    if (st == 0) {                                                             \
      if (kind == PC_SOR) memcpy(out, M, sizeof(T) * (size_t)n);               \
      else memcpy(out, f, sizeof(T) * (size_t)rp[n]);                          \
    }                                                                          \
    if (pivot) *pivot = piv;                                                   \
    free(M); free(f); free(ft); free(lo); free(up); free(rpt); free(cit);     \
    free(lot); free(upt);                                                      \
    return st;                                                                 \
  }                                                                            \
  int oracle_precond_apply_##SFX(int n, const int *rp, const int *ci,          \
                                 const T *v, int kind, double omega,           \
                                 const T *r, T *z) {                           \
    pc_##SFX pc;                                                               \
    pc_init_##SFX(&pc, kind, omega, n, rp, ci, v);                             \
    apply_##SFX(&pc, r, z);                                                    \
    pc_free_##SFX(&pc);                                                        \
    return 0;                                                                  \
  }                                                                            \
  /* equation::SOR::solve (sor.cpp:92-162) with the none preconditioner. */   \
  int oracle_sor_##SFX(int n, const int *rp, const int *ci, const T *v,        \
                       const T *b, T *x, double omega, double tol,             \
                       long maxiter, long miniter, double *hist,               \
                       long *iters, double *resid) {                           \
    T *r = calloc((size_t)n + 1, sizeof(T)), *t = calloc((size_t)n + 1, sizeof(T)); \
    T *d = NULL, *f = NULL, *ft = NULL;                                        \
    int *lo = NULL, *up = NULL, *rpt = NULL, *cit = NULL, *lot = NULL,         \
        *upt = NULL;                                                           \
    long piv;                                                                  \
    int ret = SOLVER_MAXITER;                                                  \
    long it_done = maxiter;                                                    \
    factor_build_##SFX(PC_SOR, omega, 1, n, rp, ci, v, &d, &f, &lo, &up,       \
                       &rpt, &cit, &ft, &lot, &upt, &piv);                     \
    const T bn = (T)sqrt((double)(T)DOT(n, b, b));                             \
    const T bnrm2 = (T)(1.0 / (double)bn);                                     \
    for (long iter = 0; iter < maxiter; iter++) {                              \
      spmv_##SFX(n, rp, ci, v, x, t); /* s = x (none), t = A s */              \
      for (int i = 0; i < n; i++) r[i] = b[i] - t[i];                          \
      T nrm2 = (T)sqrt((double)(T)DOT(n, r, r));                               \
      fwd_##SFX(PC_SOR, n, rp, ci, v, lo, up, d, r, t);                        \
      for (int i = 0; i < n; i++) x[i] = t[i] + x[i];                          \
      nrm2 = nrm2 * bnrm2;                                                     \
      if (hist) hist[iter] = (double)nrm2;                                     \
      if (nrm2 < tol && miniter <= iter + 1) {                                 \
        it_done = iter + 1;                                                    \
        ret = SOLVER_SUCCESS;                                                  \
        break;                                                                 \
      }                                                                        \
      if (isnan(nrm2)) {                                                       \
        it_done = iter + 1;                                                    \
        ret = SOLVER_RESIDUAL_NAN;                                             \
        break;                                                                 \
      }                                                                        \
    }                                                                          \
    if (iters) *iters = it_done;                                               \
    if (resid) *resid = (double)(T)sqrt((double)(T)DOT(n, r, r));              \
    free(r); free(t); free(d); free(f); free(ft); free(lo); free(up);         \
    free(rpt); free(cit); free(lot); free(upt);                                \
    return ret;                                                                \
  }

DEFINE_PC_EXPORTS(double, d, oracle_dot_d)
DEFINE_PC_EXPORTS(float, s, oracle_dot_s)
