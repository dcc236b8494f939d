// monolish-compatible iterative solvers on CRS (include/monolish_equation.hpp):
//   equation::CG        src/equation/cg.cpp:105-116
//   equation::BiCGSTAB  src/equation/bicgstab.cpp:155-166
//   equation::Jacobi    as a preconditioner (src/equation/jacobi.cpp:12-61)
//   equation::none      identity preconditioner (src/equation/none.cpp)
//   equation::SOR       preconditioner and solver (src/equation/sor.cpp)
//   equation::IC        IC(0) preconditioner and solve (src/equation/ic.cpp)
//   equation::ILU       ILU(0) preconditioner and solve (src/equation/ilu.cpp)
// solve(A, x, b) runs the whole Krylov loop on the device (one graph launch,
// no host round trip per iteration) and returns the reference's codes.
#pragma once
#include <cstdio>
#include <type_traits>

#include "monolish_blas.hpp"
#include "monolish_solver.hpp"
#include "monolish_vml.hpp"

namespace monolish {
namespace internal {
// kind: 0 = CG, 1 = BiCGSTAB.  Fills iters / resid; throws on library
// errors; returns the solver status.
// kind: 0 = CG, 1 = BiCGSTAB, 2 = the SOR iteration (relaxation omega);
// pc: a sweep preconditioner for CG / BiCGSTAB (nullptr: `precond`).
int krylov_solve(int kind, mlsh_csr_plan plan, const void *d_b, void *d_x, double tol,
                 size_t maxiter, size_t miniter, int precond, std::ostream *hist_out,
                 size_t *iters, double *resid, mlsh_precond pc = nullptr,
                 double omega = 1.9);
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
    // SOR / IC / ILU: the bound object's create_precond builds the device
    // preconditioner (the reference calls it at the start of every solve)
    mlsh_precond pc = nullptr;
    if (this->precond.make) pc = this->precond.make(this->precond.obj, A);
    const int st = internal::krylov_solve(
        kind, A.device_plan(), b.device_data(), x.device_data(), this->tol, this->maxiter,
        this->miniter, this->precond.kind,
        this->print_rhistory ? this->rhistory_stream : nullptr, &it, &res, pc,
        (double)this->omega);
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

// SOR, IC and ILU own a device preconditioner (mlsh_precond) built by
// create_precond and applied by apply_precond; bound to CG / BiCGSTAB it is
// applied inside the device iteration.
template <typename MATRIX, typename Float> class SweepPrecond : public solver::solver<MATRIX, Float> {
 protected:
  mlsh_precond pc = nullptr;
  void build(MATRIX &A, int kind, const char *what) {
    static_assert(std::is_same<MATRIX, matrix::CRS<Float>>::value,
                  "the B200 solve path supports matrix::CRS<T>");
    if (A.get_row() != A.get_col()) throw std::runtime_error("error A.row != A.col");
    if (!A.get_device_mem_stat())
      throw std::runtime_error(std::string(what) + " on CPU does not impl.");
    release();
    internal::check(mlsh_precond_create(internal::handle(), A.device_plan(), kind,
                                        (double)this->omega, &pc),
                    what);
    this->precond.A = &A;
  }
  void release() {
    if (pc) mlsh_precond_destroy(pc);
    pc = nullptr;
  }
  // zero pivots as src/equation/kernel/{ic,ilu}_kernel.hpp report them: the
  // float path throws, the double path prints and carries on
  void report_pivot(const char *err) {
    int64_t row = -1;
    int structural = 0;
    mlsh_precond_zero_pivot(pc, &row, &structural);
    if (row < 0) return;
    if (structural)
      std::printf("A(%d,%d) is missing\n", (int)row, (int)row);
    else
      std::printf("U(%d,%d) is zero\n", (int)row, (int)row);
    if (std::is_same<Float, float>::value) throw std::runtime_error(err);
  }

 public:
  SweepPrecond() = default;
  SweepPrecond(const SweepPrecond &) = delete;
  SweepPrecond &operator=(const SweepPrecond &) = delete;
  ~SweepPrecond() { release(); }
  [[nodiscard]] mlsh_precond native() const { return pc; }
  void apply_precond(const vector<Float> &r, vector<Float> &z) {
    if (!pc) throw std::runtime_error("error, apply_precond before create_precond");
    internal::need_device_vec(r, "apply_precond");
    internal::need_device_vec(z, "apply_precond");
    internal::check(mlsh_precond_apply(internal::handle(), pc, r.device_data(), z.device_data()),
                    "apply_precond");
  }
};

// equation::SOR (src/equation/sor.cpp): as a preconditioner M = 1/(omega
// diag(A)) with a forward and a backward sweep; solve() is the SOR
// iteration x += (D/omega + L)^{-1} (b - A x) with the relative stopping rule.
template <typename MATRIX, typename Float> class SOR : public SweepPrecond<MATRIX, Float> {
 public:
  static constexpr int precond_kind = MLSH_PRECOND_SOR;
  void create_precond(MATRIX &A) { this->build(A, MLSH_PRECOND_SOR, "SOR::create_precond"); }
  int solve(MATRIX &A, vector<Float> &x, vector<Float> &b) {
    static_assert(std::is_same<MATRIX, matrix::CRS<Float>>::value,
                  "the B200 solve path supports matrix::CRS<T>");
    if (this->lib != 0) return MONOLISH_SOLVER_NOT_IMPL;
    if (A.get_row() != A.get_col()) throw std::runtime_error("error, A.row != A.col");
    if (!A.get_device_mem_stat() || !x.get_device_mem_stat() || !b.get_device_mem_stat())
      throw std::runtime_error(
          "error, A, x and b must be device resident (util::send) for the GPU solver");
    if (x.size() != A.get_row() || b.size() != A.get_row()) return MONOLISH_SOLVER_SIZE_ERROR;
    const double t0 = internal::now_seconds();
    size_t it = 0;
    double res = 0.0;
    const int st = internal::krylov_solve(
        2, A.device_plan(), b.device_data(), x.device_data(), this->tol, this->maxiter,
        this->miniter, MLSH_PRECOND_NONE, this->print_rhistory ? this->rhistory_stream : nullptr,
        &it, &res, nullptr, (double)this->omega);
    this->final_iter = it;
    this->final_resid = res;
    internal::log_solver("solve/equation::SOR", internal::now_seconds() - t0);
    return st;
  }
  std::string name() const { return "monolish::equation::SOR"; }
  std::string solver_name() const { return "SOR"; }
};

// equation::IC (src/equation/ic.cpp): IC(0), A ~ L L^T; solve() applies it
// once (x = (L L^T)^{-1} b), as the reference's IC::solve does.
template <typename MATRIX, typename Float> class IC : public SweepPrecond<MATRIX, Float> {
 public:
  static constexpr int precond_kind = MLSH_PRECOND_IC;
  void create_precond(MATRIX &A) {
    this->build(A, MLSH_PRECOND_IC, "IC::create_precond");
    this->report_pivot("IC error.");
  }
  int solve(MATRIX &A, vector<Float> &x, vector<Float> &b) {
    create_precond(A);
    this->apply_precond(b, x);
    return MONOLISH_SOLVER_SUCCESS;
  }
  std::string name() const { return "monolish::equation::IC"; }
  std::string solver_name() const { return "IC"; }
};

// equation::ILU (src/equation/ilu.cpp): ILU(0), A ~ L U with unit L.
template <typename MATRIX, typename Float> class ILU : public SweepPrecond<MATRIX, Float> {
 public:
  static constexpr int precond_kind = MLSH_PRECOND_ILU;
  void create_precond(MATRIX &A) {
    this->build(A, MLSH_PRECOND_ILU, "ILU::create_precond");
    this->report_pivot("ILU error.");
  }
  int solve(MATRIX &A, vector<Float> &x, vector<Float> &b) {
    create_precond(A);
    this->apply_precond(b, x);
    return MONOLISH_SOLVER_SUCCESS;
  }
  std::string name() const { return "monolish::equation::ILU"; }
  std::string solver_name() const { return "ILU"; }
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
