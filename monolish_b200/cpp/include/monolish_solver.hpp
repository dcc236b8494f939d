// monolish-compatible solver base (include/monolish_solver.hpp:32-252):
// the same setters and getters; the preconditioner binding records which
// preconditioner the bound object is, and the solve runs it fused into the
// device iteration.
#pragma once
#include <cstdint>
#include <fstream>
#include <functional>
#include <iostream>
#include <string>

#include "monolish/common/monolish_common.hpp"

namespace monolish {
namespace solver {

enum class initvec_scheme { RANDOM, USER };

template <typename MATRIX, typename Float> class precondition {
 public:
  vector<Float> M;
  MATRIX *A = nullptr;
  int kind = MLSH_PRECOND_NONE;
  // SOR / IC / ILU: the bound object and how to build its device
  // preconditioner for a matrix (its create_precond)
  void *obj = nullptr;
  mlsh_precond (*make)(void *obj, MATRIX &A) = nullptr;
  void set_precond_data(vector<Float> &m) { M = m; }
  vector<Float> get_precond_data() { return M; }
};

template <typename MATRIX, typename Float> class solver {
 protected:
  int lib = 0;
  double tol = 1.0e-8;
  size_t miniter = 0;
  size_t maxiter = SIZE_MAX;
  size_t resid_method = 0;
  bool print_rhistory = false;
  std::string rhistory_file;
  std::ostream *rhistory_stream = &std::cout;
  initvec_scheme initvecscheme = initvec_scheme::RANDOM;
  double final_resid = 0;
  size_t final_iter = 0;
  Float omega = 1.9;
  int singularity = 0;
  int reorder = 3;
  precondition<MATRIX, Float> precond;

  template <class PRECOND> void bind_precond(PRECOND &p) {
    precond.kind = PRECOND::precond_kind;
    if constexpr (PRECOND::precond_kind >= MLSH_PRECOND_SOR) {
      precond.obj = &p;
      precond.make = [](void *o, MATRIX &A) -> mlsh_precond {
        auto &pp = *static_cast<PRECOND *>(o);
        pp.create_precond(A);
        return pp.native();
      };
    } else {
      precond.obj = nullptr;
      precond.make = nullptr;
    }
  }

 public:
  solver() = default;
  ~solver() {
    if (rhistory_stream != &std::cout && !rhistory_file.empty()) delete rhistory_stream;
  }

  // Bind a preconditioner (equation::Jacobi, none, SOR, IC or ILU).
  template <class PRECOND> void set_create_precond(PRECOND &p) {
    bind_precond(p);
  }
  template <class PRECOND> void set_apply_precond(PRECOND &p) {
    bind_precond(p);
  }

  void set_lib(int l) { lib = l; }
  void set_tol(double t) { tol = t; }
  void set_maxiter(size_t max) { maxiter = max; }
  void set_miniter(size_t min) { miniter = min; }
  void set_residual_method(size_t r) { resid_method = r; }
  void set_print_rhistory(bool flag) {
    print_rhistory = flag;
    rhistory_stream = &std::cout;
  }
  void set_rhistory_filename(std::string file) {
    rhistory_file = file;
    rhistory_stream = new std::ofstream(rhistory_file);
    if (rhistory_stream->fail()) throw std::runtime_error("error bad filename");
    print_rhistory = true;
  }
  void set_initvec_scheme(initvec_scheme scheme) { initvecscheme = scheme; }
  void set_omega(Float w) { omega = w; }
  void set_reorder(int r) { reorder = r; }

  [[nodiscard]] int get_lib() const { return lib; }
  [[nodiscard]] double get_tol() const { return tol; }
  [[nodiscard]] size_t get_maxiter() const { return maxiter; }
  [[nodiscard]] size_t get_miniter() const { return miniter; }
  [[nodiscard]] size_t get_residual_method() const { return resid_method; }
  bool get_print_rhistory() const { return print_rhistory; }
  initvec_scheme get_initvec_scheme() const { return initvecscheme; }
  Float get_omega() { return omega; }
  int get_reorder() { return reorder; }
  int get_singularity() { return singularity; }
  double get_final_residual() { return final_resid; }
  size_t get_final_iter() { return final_iter; }
};

}  // namespace solver
}  // namespace monolish
