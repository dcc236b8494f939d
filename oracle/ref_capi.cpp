// C entry points over the reference monolish CPU library, for the test
// harness and for the CPU baseline arm of the benchmark.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the
// reference's public headers (include/monolish_blas.hpp,
// include/monolish_equation.hpp) and linked to the reference CPU library
// built from the reference sources into oracle/_ref/.  Every call goes
// through the reference's own public API and stock OSS code path:
//   - CRS construction from raw arrays: src/utils/crs_constructor.cpp:26-43
//   - blas::matvec (OpenMP row loop): src/blas/matrix/matvec/crs_matvec.hpp:101-108
//   - blas::dot / nrm2 / axpy / xpay / axpyz: src/blas/vector/{dot,nrm2,axpy,xpay,axpyz}.hpp
//   - equation::CG::solve: src/equation/cg.cpp:13-116
//   - equation::BiCGSTAB::solve: src/equation/bicgstab.cpp:13-166
//   - equation::Jacobi as preconditioner: src/equation/jacobi.cpp:12-61
//   - equation::SOR as preconditioner and as solver: src/equation/sor.cpp
//   - blas::matvec_T, COO::sort, CRS(COO&): see the entry points below
// Nothing in the product links against this file.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <omp.h>

#include "monolish_blas.hpp"
#include "monolish_equation.hpp"
#include "monolish_vml.hpp"

namespace {

double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

template <typename T>
monolish::matrix::CRS<T> make_crs(int n, int nnz, const int *rp, const int *ci,
                                  const T *v) {
  return monolish::matrix::CRS<T>(n, n, nnz, rp, ci, v);
}

template <typename T>
int spmv_impl(int n, int nnz, const int *rp, const int *ci, const T *v,
              const T *x, T *y, int reps, double *seconds) {
  auto A = make_crs<T>(n, nnz, rp, ci, v);
  monolish::vector<T> xv(x, x + n);
  monolish::vector<T> yv(n, 0.0);
  double best = 1e300, total = 0.0;
  int r = reps < 1 ? 1 : reps;
  for (int i = 0; i < r; ++i) {
    double t0 = now_s();
    monolish::blas::matvec(A, xv, yv);
    double dt = now_s() - t0;
    total += dt;
    if (dt < best) best = dt;
  }
  std::memcpy(y, yv.data(), sizeof(T) * n);
  if (seconds) {
    seconds[0] = total / r;
    seconds[1] = best;
  }
  return 0;
}

// Runs one solve through the reference's public solver API, exactly as the
// reference's test harness test/equation/iterative/equation_kernel.hpp:5-57
// wires it (set_tol / set_maxiter / set_miniter / set_create_precond /
// set_apply_precond / solve).
template <typename T, typename SOLVER>
int solve_impl(int n, int nnz, const int *rp, const int *ci, const T *v,
               const T *b, T *x, double tol_abs, long maxiter, int precond,
               long *iters, double *resid, double *seconds) {
  auto A = make_crs<T>(n, nnz, rp, ci, v);
  monolish::vector<T> bv(b, b + n);
  monolish::vector<T> xv(x, x + n);
  SOLVER solver;
  solver.set_tol(tol_abs);
  solver.set_lib(0);
  solver.set_miniter(0);
  solver.set_maxiter(static_cast<size_t>(maxiter));
  monolish::equation::Jacobi<monolish::matrix::CRS<T>, T> jac;
  monolish::equation::SOR<monolish::matrix::CRS<T>, T> sor;
  monolish::equation::none<monolish::matrix::CRS<T>, T> non;
  if (precond == 1) {
    solver.set_create_precond(jac);
    solver.set_apply_precond(jac);
  } else if (precond == 2) {
    solver.set_create_precond(sor);
    solver.set_apply_precond(sor);
  } else {
    solver.set_create_precond(non);
    solver.set_apply_precond(non);
  }
  double t0 = now_s();
  int ret = solver.solve(A, xv, bv);
  double dt = now_s() - t0;
  std::memcpy(x, xv.data(), sizeof(T) * n);
  if (iters) *iters = static_cast<long>(solver.get_final_iter());
  if (resid) *resid = solver.get_final_residual();
  if (seconds) *seconds = dt;
  return ret;
}

// equation::SOR::solve (src/equation/sor.cpp:92-162) with the default
// none preconditioner.
template <typename T>
int sor_solve_impl(int n, int nnz, const int *rp, const int *ci, const T *v, const T *b, T *x,
                   double omega, double tol, long maxiter, long *iters, double *resid,
                   double *seconds) {
  auto A = make_crs<T>(n, nnz, rp, ci, v);
  monolish::vector<T> bv(b, b + n);
  monolish::vector<T> xv(x, x + n);
  monolish::equation::SOR<monolish::matrix::CRS<T>, T> solver;
  monolish::equation::none<monolish::matrix::CRS<T>, T> non;
  solver.set_tol(tol);
  solver.set_lib(0);
  solver.set_miniter(0);
  solver.set_maxiter(static_cast<size_t>(maxiter));
  solver.set_omega(static_cast<T>(omega));
  solver.set_create_precond(non);
  solver.set_apply_precond(non);
  double t0 = now_s();
  int ret = solver.solve(A, xv, bv);
  double dt = now_s() - t0;
  std::memcpy(x, xv.data(), sizeof(T) * n);
  if (iters) *iters = static_cast<long>(solver.get_final_iter());
  if (resid) *resid = solver.get_final_residual();
  if (seconds) *seconds = dt;
  return ret;
}

// equation::SOR::create_precond + apply_precond (sor.cpp:13-69).
template <typename T>
int sor_apply_impl(int n, int nnz, const int *rp, const int *ci, const T *v, double omega,
                   const T *r, T *z) {
  auto A = make_crs<T>(n, nnz, rp, ci, v);
  monolish::vector<T> rv(r, r + n);
  monolish::vector<T> zv(n, 0.0);
  monolish::equation::SOR<monolish::matrix::CRS<T>, T> pc;
  pc.set_omega(static_cast<T>(omega));
  pc.create_precond(A);
  pc.apply_precond(rv, zv);
  std::memcpy(z, zv.data(), sizeof(T) * n);
  return 0;
}

} // namespace

extern "C" {

int ref_sor_d(int n, int nnz, const int *rp, const int *ci, const double *v, const double *b,
              double *x, double omega, double tol, long maxiter, long *iters, double *resid,
              double *seconds) {
  return sor_solve_impl<double>(n, nnz, rp, ci, v, b, x, omega, tol, maxiter, iters, resid,
                                seconds);
}
int ref_sor_s(int n, int nnz, const int *rp, const int *ci, const float *v, const float *b,
              float *x, double omega, double tol, long maxiter, long *iters, double *resid,
              double *seconds) {
  return sor_solve_impl<float>(n, nnz, rp, ci, v, b, x, omega, tol, maxiter, iters, resid,
                               seconds);
}
int ref_sor_apply_d(int n, int nnz, const int *rp, const int *ci, const double *v,
                    double omega, const double *r, double *z) {
  return sor_apply_impl<double>(n, nnz, rp, ci, v, omega, r, z);
}
int ref_sor_apply_s(int n, int nnz, const int *rp, const int *ci, const float *v,
                    double omega, const float *r, float *z) {
  return sor_apply_impl<float>(n, nnz, rp, ci, v, omega, r, z);
}

// y = A^T x through blas::matvec_T (src/blas/matrix/matvec/crs_matvec.hpp:88-98
// for the OSS path) on an n_rows x n_cols CRS<double>.
int ref_spmv_t_d(int n_rows, int n_cols, int nnz, const int *rp, const int *ci,
                 const double *v, const double *x, double *y) {
  monolish::matrix::CRS<double> A(n_rows, n_cols, nnz, rp, ci, v);
  monolish::vector<double> xv(x, x + n_rows);
  monolish::vector<double> yv(n_cols, 0.0);
  monolish::blas::matvec_T(A, xv, yv);
  std::memcpy(y, yv.data(), sizeof(double) * n_cols);
  return 0;
}

// COO<double>::sort(merge) (src/utils/at_insert_sort/at_insert_sort_coo.cpp:119-145)
// on a COO built from raw arrays; the sorted entries are written back and
// their count returned.
long ref_coo_sort_d(int n_rows, int n_cols, long nnz, int *row, int *col, double *val,
                    int merge) {
  monolish::matrix::COO<double> A(n_rows, n_cols, nnz, row, col, val);
  A.sort(merge != 0);
  const long out = (long)A.get_nnz();
  std::memcpy(row, A.row_index.data(), sizeof(int) * out);
  std::memcpy(col, A.col_index.data(), sizeof(int) * out);
  std::memcpy(val, A.data(), sizeof(double) * out);
  return out;
}

// CRS<double>(COO&) (src/utils/convert/convert_crs.cpp:9-43): the row
// pointer built from a row-sorted COO.
int ref_coo_to_crs_d(int n_rows, int n_cols, long nnz, const int *row, const int *col,
                     const double *val, int *rp) {
  monolish::matrix::COO<double> A(n_rows, n_cols, nnz, row, col, val);
  monolish::matrix::CRS<double> B(A);
  std::memcpy(rp, B.row_ptr.data(), sizeof(int) * (n_rows + 1));
  return 0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }
void ref_set_threads(int n) { omp_set_num_threads(n); }

int ref_spmv_d(int n, int nnz, const int *rp, const int *ci, const double *v,
               const double *x, double *y, int reps, double *seconds) {
  return spmv_impl<double>(n, nnz, rp, ci, v, x, y, reps, seconds);
}
int ref_spmv_s(int n, int nnz, const int *rp, const int *ci, const float *v,
               const float *x, float *y, int reps, double *seconds) {
  return spmv_impl<float>(n, nnz, rp, ci, v, x, y, reps, seconds);
}

int ref_cg_d(int n, int nnz, const int *rp, const int *ci, const double *v,
             const double *b, double *x, double tol_abs, long maxiter,
             int precond, long *iters, double *resid, double *seconds) {
  using S = monolish::equation::CG<monolish::matrix::CRS<double>, double>;
  return solve_impl<double, S>(n, nnz, rp, ci, v, b, x, tol_abs, maxiter,
                               precond, iters, resid, seconds);
}
int ref_cg_s(int n, int nnz, const int *rp, const int *ci, const float *v,
             const float *b, float *x, double tol_abs, long maxiter,
             int precond, long *iters, double *resid, double *seconds) {
  using S = monolish::equation::CG<monolish::matrix::CRS<float>, float>;
  return solve_impl<float, S>(n, nnz, rp, ci, v, b, x, tol_abs, maxiter,
                              precond, iters, resid, seconds);
}
int ref_bicgstab_d(int n, int nnz, const int *rp, const int *ci,
                   const double *v, const double *b, double *x, double tol_abs,
                   long maxiter, int precond, long *iters, double *resid,
                   double *seconds) {
  using S = monolish::equation::BiCGSTAB<monolish::matrix::CRS<double>, double>;
  return solve_impl<double, S>(n, nnz, rp, ci, v, b, x, tol_abs, maxiter,
                               precond, iters, resid, seconds);
}
int ref_bicgstab_s(int n, int nnz, const int *rp, const int *ci,
                   const float *v, const float *b, float *x, double tol_abs,
                   long maxiter, int precond, long *iters, double *resid,
                   double *seconds) {
  using S = monolish::equation::BiCGSTAB<monolish::matrix::CRS<float>, float>;
  return solve_impl<float, S>(n, nnz, rp, ci, v, b, x, tol_abs, maxiter,
                              precond, iters, resid, seconds);
}

// Vector BLAS through the reference's public API (host-resident vectors).
double ref_dot_d(long n, const double *x, const double *y) {
  monolish::vector<double> a(x, x + n), b(y, y + n);
  return monolish::blas::dot(a, b);
}
double ref_nrm2_d(long n, const double *x) {
  monolish::vector<double> a(x, x + n);
  return monolish::blas::nrm2(a);
}
void ref_axpy_d(long n, double alpha, const double *x, double *y) {
  monolish::vector<double> a(x, x + n), b(y, y + n);
  monolish::blas::axpy(alpha, a, b);
  std::memcpy(y, b.data(), sizeof(double) * n);
}
void ref_xpay_d(long n, double alpha, const double *x, double *y) {
  monolish::vector<double> a(x, x + n), b(y, y + n);
  monolish::blas::xpay(alpha, a, b);
  std::memcpy(y, b.data(), sizeof(double) * n);
}
void ref_axpyz_d(long n, double alpha, const double *x, const double *y,
                 double *z) {
  monolish::vector<double> a(x, x + n), b(y, y + n), c(n, 0.0);
  monolish::blas::axpyz(alpha, a, b, c);
  std::memcpy(z, c.data(), sizeof(double) * n);
}
// The reference's seeded random vector constructor
// (src/utils/vector_constructor.cpp:98-110).
void ref_random_vector_d(long n, double lo, double hi, unsigned seed,
                         double *out) {
  monolish::vector<double> a(static_cast<size_t>(n), lo, hi, seed);
  std::memcpy(out, a.data(), sizeof(double) * n);
}
// The reference's 2D 5-point generator (src/utils/create_matrix/laplacian_2D5p.cpp)
// converted to CRS (src/utils/convert/convert_crs.cpp:9-43); fills the
// caller's arrays (row_ptr n+1, col/val nnz) and returns nnz, or the nnz
// needed when the arrays are NULL.
long ref_laplacian_2d5p_d(int m, int n, int *rp, int *ci, double *v) {
  auto coo = monolish::util::laplacian_matrix_2D_5p<double>(m, n);
  monolish::matrix::CRS<double> A(coo);
  long nnz = static_cast<long>(A.get_nnz());
  if (rp && ci && v) {
    std::memcpy(rp, A.row_ptr.data(), sizeof(int) * (A.get_row() + 1));
    std::memcpy(ci, A.col_ind.data(), sizeof(int) * nnz);
    std::memcpy(v, A.data(), sizeof(double) * nnz);
  }
  return nnz;
}

} // extern "C"
