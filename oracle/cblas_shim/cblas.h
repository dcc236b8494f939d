/*
 * Minimal CBLAS interface for building the reference monolish CPU library
 * against the OpenBLAS build that SciPy bundles (its exports carry a
 * `scipy_` prefix).  Only the routines the reference library calls are
 * declared; each is mapped onto the prefixed export.
 *
 * Test infrastructure only: used by oracle/Makefile to build the reference
 * into oracle/_ref/.  Nothing in the product links against it.
 */
#ifndef MLSH_ORACLE_CBLAS_SHIM_H
#define MLSH_ORACLE_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum {
  CblasNoTrans = 111,
  CblasTrans = 112,
  CblasConjTrans = 113
} CBLAS_TRANSPOSE;

#define cblas_ddot scipy_cblas_ddot
#define cblas_sdot scipy_cblas_sdot
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_saxpy scipy_cblas_saxpy
#define cblas_dcopy scipy_cblas_dcopy
#define cblas_scopy scipy_cblas_scopy
#define cblas_dscal scipy_cblas_dscal
#define cblas_sscal scipy_cblas_sscal
#define cblas_dasum scipy_cblas_dasum
#define cblas_sasum scipy_cblas_sasum
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_sgemv scipy_cblas_sgemv
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_sgemm scipy_cblas_sgemm

typedef int blasint;

double cblas_ddot(const blasint n, const double *x, const blasint incx,
                  const double *y, const blasint incy);
float cblas_sdot(const blasint n, const float *x, const blasint incx,
                 const float *y, const blasint incy);
void cblas_daxpy(const blasint n, const double alpha, const double *x,
                 const blasint incx, double *y, const blasint incy);
void cblas_saxpy(const blasint n, const float alpha, const float *x,
                 const blasint incx, float *y, const blasint incy);
void cblas_dcopy(const blasint n, const double *x, const blasint incx,
                 double *y, const blasint incy);
void cblas_scopy(const blasint n, const float *x, const blasint incx, float *y,
                 const blasint incy);
void cblas_dscal(const blasint n, const double alpha, double *x,
                 const blasint incx);
void cblas_sscal(const blasint n, const float alpha, float *x,
                 const blasint incx);
double cblas_dasum(const blasint n, const double *x, const blasint incx);
float cblas_sasum(const blasint n, const float *x, const blasint incx);
void cblas_dgemv(const CBLAS_ORDER order, const CBLAS_TRANSPOSE trans,
                 const blasint m, const blasint n, const double alpha,
                 const double *a, const blasint lda, const double *x,
                 const blasint incx, const double beta, double *y,
                 const blasint incy);
void cblas_sgemv(const CBLAS_ORDER order, const CBLAS_TRANSPOSE trans,
                 const blasint m, const blasint n, const float alpha,
                 const float *a, const blasint lda, const float *x,
                 const blasint incx, const float beta, float *y,
                 const blasint incy);
void cblas_dgemm(const CBLAS_ORDER order, const CBLAS_TRANSPOSE transa,
                 const CBLAS_TRANSPOSE transb, const blasint m,
                 const blasint n, const blasint k, const double alpha,
                 const double *a, const blasint lda, const double *b,
                 const blasint ldb, const double beta, double *c,
                 const blasint ldc);
void cblas_sgemm(const CBLAS_ORDER order, const CBLAS_TRANSPOSE transa,
                 const CBLAS_TRANSPOSE transb, const blasint m,
                 const blasint n, const blasint k, const float alpha,
                 const float *a, const blasint lda, const float *b,
                 const blasint ldb, const float beta, float *c,
                 const blasint ldc);

#ifdef __cplusplus
}
#endif

#endif
