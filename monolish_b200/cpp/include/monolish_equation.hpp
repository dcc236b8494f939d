// monolish-compatible iterative solvers on CRS (include/monolish_equation.hpp):
//   equation::CG        src/equation/cg.cpp:105-116
//   equation::BiCGSTAB  src/equation/bicgstab.cpp:155-166
//   equation::Jacobi    as a preconditioner (src/equation/jacobi.cpp:12-61)
//   equation::none      identity preconditioner (src/equation/none.cpp)
// solve(A, x, b) runs the whole Krylov loop on the device (one graph launch,
// no host round trip per iteration) and returns the reference's codes.
#pragma once
#include <type_traits>

#include "monolish_blas.hpp"
#include "monolish_solver.hpp"
#include "monolish_vml.hpp"

namespace monolish {
namespace internal {
// kind: 0 = CG, 1 = BiCGSTAB.  Fills iters / resid; throws on library
// errors; returns the solver status.
int krylov_solve(int kind, mlsh_csr_plan plan, const void *d_b, void *d_x, double tol,
                 size_t maxiter, size_t miniter, int precond, std::ostream *hist_out,
                 size_t *iters, double *resid);
void log_solver(const char *name, double seconds);
double now_seconds();
}  // namespace internal

namespace equation {

template <typename MATRIX, typename Float> class Krylov : public solver::solver<MATRIX, Float> {
 protected:
  int run(int kind, const char *name, MATRIX &A, vector<Float> &x, vector<Float> &b) {
    static_assert(std::is_same<MATRIX, matrix::CRS<Float>>::value,
                  "the B200 solve path supports matrix::CRS<T>");
    if (A.get_row() != A.get_col()) throw std::runtime_error("error, A.row != A.col");
    if (!A.get_device_mem_stat() || !x.get_device_mem_stat() || !b.get_device_mem_stat())
      throw std::runtime_error(
          "error, A, x and b must be device resident (util::send) for the GPU solver");
    if (x.size() != A.get_row() || b.size() != A.get_row())
      return MONOLISH_SOLVER_SIZE_ERROR;
    const double t0 = internal::now_seconds();
    size_t it = 0;
    double res = 0.0;
    const int st = internal::krylov_solve(
        kind, A.device_plan(), b.device_data(), x.device_data(), this->tol, this->maxiter,
        this->miniter, this->precond.kind,
        this->print_rhistory ? this->rhistory_stream : nullptr, &it, &res);
    this->final_iter = it;
    this->final_resid = res;
    internal::log_solver(name, internal::now_seconds() - t0);
    return st;
  }
};

template <typename MATRIX, typename Float> class CG : public Krylov<MATRIX, Float> {
 public:
  int solve(MATRIX &A, vector<Float> &x, vector<Float> &b) {
    if (this->lib != 0) return MONOLISH_SOLVER_NOT_IMPL;
    return this->run(0, "solve/equation::CG", A, x, b);
  }
  std::string name() const { return "monolish_equation_CG"; }
  std::string solver_name() const { return "CG"; }
};

template <typename MATRIX, typename Float> class BiCGSTAB : public Krylov<MATRIX, Float> {
 public:
  int solve(MATRIX &A, vector<Float> &x, vector<Float> &b) {
    if (this->lib != 0) return MONOLISH_SOLVER_NOT_IMPL;
    return this->run(1, "solve/equation::BiCGSTAB", A, x, b);
  }
  std::string name() const { return "monolish_equation_BiCGSTAB"; }
  std::string solver_name() const { return "BiCGSTAB"; }
};

// Jacobi: as a preconditioner it is fused into the device iteration; its
// standalone create/apply are also provided.  The stationary Jacobi solver
// itself is not part of this path (solve returns NOT_IMPL).
template <typename MATRIX, typename Float> class Jacobi : public solver::solver<MATRIX, Float> {
 public:
  static constexpr int precond_kind = MLSH_PRECOND_JACOBI;
  void create_precond(MATRIX &A) {
    if (A.get_row() != A.get_col()) throw std::runtime_error("error A.row != A.col");
    this->precond.M = vector<Float>(A.get_row(), 0.0);
    this->precond.M.send();
    A.diag(this->precond.M);
    vml::reciprocal(this->precond.M, this->precond.M);
  }
  void apply_precond(const vector<Float> &r, vector<Float> &z) {
    vml::mul(this->precond.M, r, z);
  }
  int solve(MATRIX &, vector<Float> &, vector<Float> &) { return MONOLISH_SOLVER_NOT_IMPL; }
  std::string name() const { return "monolish_equation_Jacobi"; }
  std::string solver_name() const { return "Jacobi"; }
};

template <typename MATRIX, typename Float> class none : public solver::solver<MATRIX, Float> {
 public:
  static constexpr int precond_kind = MLSH_PRECOND_NONE;
  void create_precond(MATRIX &) {}
  void apply_precond(const vector<Float> &r, vector<Float> &z) { blas::copy(r, z); }
  int solve(MATRIX &, vector<Float> &, vector<Float> &) { return MONOLISH_SOLVER_SUCCESS; }
  std::string name() const { return "monolish_equation_none"; }
  std::string solver_name() const { return "none"; }
};

}  // namespace equation
}  // namespace monolish
