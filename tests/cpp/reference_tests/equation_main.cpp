// Runs the reference's solver test (test/equation/iterative/
// equation_kernel.hpp, used unchanged) against this library's C++ layer:
// CG and BiCGSTAB on CRS<double> / CRS<float>, without a preconditioner
// and with Jacobi, on the matrix file given (the reference's test.mtx), the
// answer checked as the reference checks it (x vs ones, tol * 10).
#include "equation_kernel.hpp"

#include <cstdlib>

template <template <typename, typename> class SOLVER, template <typename, typename> class PC>
bool both(const char *file, int check, const char *name) {
  using namespace monolish;
  std::cout << "CRS, " << name << std::endl;
  return test<matrix::CRS<double>, double, SOLVER<matrix::CRS<double>, double>,
              PC<matrix::CRS<double>, double>>(file, check, 1.0e-8) &&
         test<matrix::CRS<float>, float, SOLVER<matrix::CRS<float>, float>,
              PC<matrix::CRS<float>, float>>(file, check, 1.0e-4);
}

int main(int argc, char **argv) {
  if (argc != 3) {
    std::cout << "usage: " << argv[0] << " matrix.mtx check(1/0)" << std::endl;
    return 1;
  }
  using namespace monolish::equation;
  const char *file = argv[1];
  const int check = std::atoi(argv[2]);
  const bool ok = both<CG, none>(file, check, "CG, none") &&
                  both<CG, Jacobi>(file, check, "CG, Jacobi") &&
                  both<BiCGSTAB, none>(file, check, "BiCGSTAB, none") &&
                  both<BiCGSTAB, Jacobi>(file, check, "BiCGSTAB, Jacobi");
  std::cout << (ok ? "PASS" : "FAIL") << std::endl;
  return ok ? 0 : 1;
}
