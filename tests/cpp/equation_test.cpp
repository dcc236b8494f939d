// Solver test written against the monolish API (CRS + vector + send +
// equation::CG/BiCGSTAB with none/Jacobi/SOR/IC/ILU, the SOR solver and the
// sparse IC / ILU solves), built against the B200 drop-in headers.  It
// follows the reference's own solver test flow
// (test/equation/iterative/equation_kernel.hpp): read a MatrixMarket matrix,
// b = A*ones, x0 = seeded U(0,1), solve, check x against ones at tol*10.
//
// usage: equation_test <matrix.mtx>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <random>

#include "monolish_blas.hpp"
#include "monolish_equation.hpp"

namespace {

std::mt19937 engine(1234);

template <typename T> bool close_to_ones(const monolish::vector<T> &x, double tol) {
  for (size_t i = 0; i < x.size(); ++i) {
    const double d = std::fabs((double)x.data()[i] - 1.0);
    if (d > tol && d > tol * 1.0) {
      std::cout << "  x[" << i << "] = " << x.data()[i] << std::endl;
      return false;
    }
  }
  return true;
}

template <typename T, typename SOLVER, typename PRECOND>
bool run(const char *file, double tol, const char *label, double xtol = -1.0) {
  monolish::matrix::COO<T> coo(file);
  monolish::matrix::CRS<T> A(coo);
  monolish::vector<T> ones(A.get_row(), 1.0);
  monolish::vector<T> b(A.get_row(), 0.0);
  monolish::vector<T> x(A.get_row(), 0.0, 1.0, engine());
  monolish::util::send(A, x, b, ones);
  monolish::blas::matvec(A, ones, b);

  SOLVER solver;
  solver.set_tol(tol);
  solver.set_lib(0);
  solver.set_miniter(0);
  solver.set_maxiter(10000);
  PRECOND precond;
  solver.set_create_precond(precond);
  solver.set_apply_precond(precond);
  const int st = solver.solve(A, x, b);
  x.recv();
  std::cout << label << ": status " << st << ", iter " << solver.get_final_iter()
            << ", resid " << solver.get_final_residual() << std::endl;
  if (st != MONOLISH_SOLVER_SUCCESS) return false;
  return close_to_ones(x, xtol > 0 ? xtol : tol * 10);
}

// test/equation/sparse_ic, sparse_ilu: x = M^{-1} b with b = A*ones; exact
// where the incomplete factorization is exact (a tridiagonal matrix).
template <typename T, typename SOLVER> bool run_direct(const char *file, double tol,
                                                       const char *label) {
  monolish::matrix::COO<T> coo(file);
  monolish::matrix::CRS<T> A(coo);
  monolish::vector<T> ones(A.get_row(), 1.0);
  monolish::vector<T> b(A.get_row(), 0.0);
  monolish::vector<T> x(A.get_row(), 0.0, 1.0, engine());
  monolish::util::send(A, x, b, ones);
  monolish::blas::matvec(A, ones, b);
  SOLVER solver;
  const int st = solver.solve(A, x, b);
  x.recv();
  std::cout << label << ": status " << st << std::endl;
  return st == MONOLISH_SOLVER_SUCCESS && close_to_ones(x, tol);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 2) {
    std::cerr << "usage: equation_test <matrix.mtx>" << std::endl;
    return 2;
  }
  using namespace monolish;
  const char *f = argv[1];
  using CD = matrix::CRS<double>;
  using CF = matrix::CRS<float>;
  bool ok = true;
  ok &= run<double, equation::CG<CD, double>, equation::none<CD, double>>(f, 1e-8, "CG none d");
  ok &= run<float, equation::CG<CF, float>, equation::none<CF, float>>(f, 1e-4, "CG none f");
  ok &= run<double, equation::CG<CD, double>, equation::Jacobi<CD, double>>(f, 1e-8, "CG Jacobi d");
  ok &= run<float, equation::CG<CF, float>, equation::Jacobi<CF, float>>(f, 1e-4, "CG Jacobi f");
  ok &= run<double, equation::BiCGSTAB<CD, double>, equation::none<CD, double>>(
      f, 1e-8, "BiCGSTAB none d");
  ok &= run<float, equation::BiCGSTAB<CF, float>, equation::none<CF, float>>(
      f, 1e-4, "BiCGSTAB none f");
  ok &= run<double, equation::BiCGSTAB<CD, double>, equation::Jacobi<CD, double>>(
      f, 1e-8, "BiCGSTAB Jacobi d");
  ok &= run<float, equation::BiCGSTAB<CF, float>, equation::Jacobi<CF, float>>(
      f, 1e-4, "BiCGSTAB Jacobi f");
  // the sweep preconditioners (test/equation/iterative/{cg,bicgstab}.cpp)
  ok &= run<double, equation::CG<CD, double>, equation::SOR<CD, double>>(f, 1e-8, "CG SOR d");
  ok &= run<float, equation::CG<CF, float>, equation::SOR<CF, float>>(f, 1e-4, "CG SOR f");
  ok &= run<double, equation::CG<CD, double>, equation::IC<CD, double>>(f, 1e-8, "CG IC d");
  ok &= run<float, equation::CG<CF, float>, equation::IC<CF, float>>(f, 1e-4, "CG IC f");
  ok &= run<double, equation::CG<CD, double>, equation::ILU<CD, double>>(f, 1e-8, "CG ILU d");
  ok &= run<float, equation::CG<CF, float>, equation::ILU<CF, float>>(f, 1e-4, "CG ILU f");
  ok &= run<double, equation::BiCGSTAB<CD, double>, equation::SOR<CD, double>>(
      f, 1e-8, "BiCGSTAB SOR d");
  ok &= run<double, equation::BiCGSTAB<CD, double>, equation::IC<CD, double>>(
      f, 1e-8, "BiCGSTAB IC d");
  ok &= run<double, equation::BiCGSTAB<CD, double>, equation::ILU<CD, double>>(
      f, 1e-8, "BiCGSTAB ILU d");
  // on the 3x3 tridiagonal matrix ILU(0) is exact: in FP32 the first s =
  // r - alpha v is exactly 0 and omega = (t,s)/(t,t) = 0/0, so the
  // reference's recurrence (bicgstab.cpp:91-102) ends with a NaN residual
  // there; the case runs on the larger matrix only
  const bool tridiag3 = matrix::COO<double>(f).get_row() == 3;
  if (!tridiag3)
    ok &= run<float, equation::BiCGSTAB<CF, float>, equation::ILU<CF, float>>(
        f, 1e-4, "BiCGSTAB ILU f");
  // the SOR iteration itself (test/equation/iterative/sor.cpp); its test is
  // relative, so x is checked at the accuracy that implies here
  ok &= run<double, equation::SOR<CD, double>, equation::none<CD, double>>(f, 1e-8, "SOR d",
                                                                            1e-5);
  ok &= run<float, equation::SOR<CF, float>, equation::none<CF, float>>(f, 1e-4, "SOR f", 1e-2);
  if (monolish::util::build_with_gpu()) {
    if (tridiag3) {  // the reference's tridiagonal test matrix
      ok &= run_direct<double, equation::IC<CD, double>>(f, 1e-8, "IC solve d");
      ok &= run_direct<float, equation::IC<CF, float>>(f, 1e-5, "IC solve f");
      ok &= run_direct<double, equation::ILU<CD, double>>(f, 1e-8, "ILU solve d");
      ok &= run_direct<float, equation::ILU<CF, float>>(f, 1e-5, "ILU solve f");
    }
  }
  std::cout << (ok ? "PASS" : "FAIL") << std::endl;
  return ok ? 0 : 1;
}
