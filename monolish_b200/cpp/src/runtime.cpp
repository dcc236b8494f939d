// Runtime of the monolish-compatible C++ layer: the per-thread handle,
// error mapping, device residency helpers, BLAS/VML entry points, COO
// construction and MatrixMarket input, the solver driver and the logger.
// Every numerical operation is a call into the CUDA library (include/mlsh.h).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "monolish_blas.hpp"
#include "monolish_equation.hpp"
#include "monolish_vml.hpp"

namespace monolish {

// ================================================================ internal
namespace internal {

namespace {
struct HandleOwner {
  mlsh_handle h = nullptr;
  ~HandleOwner() {
    if (h) mlsh_destroy(h);
  }
};
thread_local HandleOwner t_handle;

struct LogState {
  size_t level = 0;
  std::string file;
  std::mutex mu;
};
LogState &log_state() {
  static LogState s;
  return s;
}
}  // namespace

mlsh_handle handle() {
  if (!t_handle.h) {
    const int st = mlsh_create(&t_handle.h);
    if (st != MLSH_SUCCESS)
      throw std::runtime_error(std::string("monolish_b200: cannot create device handle: ") +
                               mlsh_status_string(st));
  }
  return t_handle.h;
}

void check(int status, const char *what) {
  if (status >= MONOLISH_SOLVER_NOT_IMPL) return;  // success or a solver code
  throw std::runtime_error(std::string("monolish_b200: ") + what + ": " +
                           mlsh_status_string(status) + " " + mlsh_last_error());
}

void *dalloc(size_t bytes) {
  void *p = nullptr;
  check(mlsh_device_alloc(bytes, &p), "device allocation");
  return p;
}
void dfree(void *p) {
  if (p) mlsh_device_free(p);
}
void h2d(void *d, const void *h, size_t bytes) {
  check(mlsh_memcpy_h2d(handle(), d, h, bytes), "send");
}
void d2h(void *h, const void *d, size_t bytes) {
  check(mlsh_memcpy_d2h(handle(), h, d, bytes), "recv");
}
void d2d(void *d, const void *s, size_t bytes) {
  check(mlsh_memcpy_d2d(handle(), d, s, bytes), "device copy");
}

double now_seconds() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

void log_solver(const char *name, double seconds) {
  LogState &s = log_state();
  if (s.level < 1) return;
  std::lock_guard<std::mutex> lk(s.mu);
  std::ostringstream line;
  line << "- {type : solver, name : " << name << ", time : " << std::setprecision(9) << seconds
       << "}\n";
  if (s.file.empty()) {
    std::cout << line.str();
  } else {
    std::ofstream out(s.file, std::ios::app);
    out << line.str();
  }
}

int krylov_solve(int kind, mlsh_csr_plan plan, const void *d_b, void *d_x, double tol,
                 size_t maxiter, size_t miniter, int precond, std::ostream *hist_out,
                 size_t *iters, double *resid, mlsh_precond pc, double omega) {
  mlsh_solver_opts o;
  mlsh_solver_opts_default(&o);
  o.tol = tol;
  o.maxiter = maxiter > (size_t)INT64_MAX ? INT64_MAX : (int64_t)maxiter;
  o.miniter = miniter > (size_t)INT64_MAX ? INT64_MAX : (int64_t)miniter;
  o.precond = precond;
  std::vector<double> hist;
  if (hist_out) {
    const int64_t cap = std::min<int64_t>(o.maxiter, int64_t(1) << 22);
    hist.assign((size_t)std::max<int64_t>(cap, 1), 0.0);
    o.history = hist.data();
    o.history_len = cap;
  }
  mlsh_solver_result r{};
  int st;
  if (kind == 2) {  // the SOR iteration (its own preconditioner: none)
    o.precond = MLSH_PRECOND_NONE;
    st = mlsh_sor_solve(handle(), plan, d_b, d_x, omega, &o, &r);
  } else if (pc) {
    st = kind == 0 ? mlsh_cg_solve_precond(handle(), plan, pc, d_b, d_x, &o, &r)
                   : mlsh_bicgstab_solve_precond(handle(), plan, pc, d_b, d_x, &o, &r);
  } else {
    st = kind == 0 ? mlsh_cg_solve(handle(), plan, d_b, d_x, &o, &r)
                   : mlsh_bicgstab_solve(handle(), plan, d_b, d_x, &o, &r);
  }
  check(st, kind == 0 ? "CG" : (kind == 1 ? "BiCGSTAB" : "SOR"));
  *iters = (size_t)r.iters;
  *resid = r.final_resid;
  if (hist_out) {
    const int64_t k = std::min<int64_t>(r.iters, o.history_len);
    for (int64_t i = 0; i < k; ++i)
      *hist_out << i + 1 << "\t" << std::scientific << hist[(size_t)i] << std::endl;
  }
  return st;
}

}  // namespace internal

// ==================================================================== util
namespace util {
void set_log_level(size_t level) { internal::log_state().level = level; }
void set_log_filename(std::string filename) { internal::log_state().file = filename; }
bool build_with_gpu() { return true; }
bool solver_check(const int err) {
  (void)err;
  return false;
}

template <typename T> matrix::COO<T> laplacian_matrix_2D_5p(const int m, const int n) {
  const int size = m * n;
  matrix::COO<T> mat(size, size);
  for (int ii = 0; ii < size; ii++) {
    const int i = ii / m;
    const int j = ii - i * m;
    if (i > 0) mat.insert(ii, ii - m, -1.0);
    if (j > 0) mat.insert(ii, ii - 1, -1.0);
    mat.insert(ii, ii, 4.0);
    if (j < m - 1) mat.insert(ii, ii + 1, -1.0);
    if (i < n - 1) mat.insert(ii, ii + m, -1.0);
  }
  return mat;
}
template matrix::COO<double> laplacian_matrix_2D_5p<double>(const int, const int);
template matrix::COO<float> laplacian_matrix_2D_5p<float>(const int, const int);
}  // namespace util

// ===================================================================== COO
namespace matrix {

template <typename Float> void COO<Float>::input_mm(const std::string filename) {
  std::ifstream ifs(filename);
  if (!ifs) throw std::runtime_error("Matrix.input: cannot open file " + filename);
  std::string banner;
  std::getline(ifs, banner);
  std::istringstream bn(banner);
  std::string mm, mat, fmt, dtype, dstruct;
  bn >> mm >> mat >> fmt >> dtype >> dstruct;
  if (mm != "%%MatrixMarket" || mat != "matrix" || fmt != "coordinate")
    throw std::runtime_error("Matrix.input: not a MatrixMarket coordinate matrix: " + filename);
  if (dtype != "real" && dtype != "double" && dtype != "integer")
    throw std::runtime_error("Matrix.input: unsupported value type " + dtype);
  if (dstruct != "general")
    throw std::runtime_error("Matrix.input: unsupported structure " + dstruct);
  std::string line;
  while (std::getline(ifs, line))
    if (!line.empty() && line[0] != '%') break;
  std::istringstream hdr(line);
  size_t M = 0, N = 0, NNZ = 0;
  hdr >> M >> N >> NNZ;
  rowN = M;
  colN = N;
  row_index.resize(NNZ);
  col_index.resize(NNZ);
  val.resize(NNZ);
  for (size_t k = 0; k < NNZ; ++k) {
    long r, c;
    double v;
    if (!(ifs >> r >> c >> v)) throw std::runtime_error("Matrix.input: truncated " + filename);
    row_index[k] = (int)(r - 1);
    col_index[k] = (int)(c - 1);
    val[k] = (Float)v;
  }
}

// COO::sort (src/utils/at_insert_sort/at_insert_sort_coo.cpp:119-145) on
// the device: the entries are copied up, sorted by (row, col) -- equal
// (row, col) keeping their input order -- and, with merge, each such run
// collapses to one entry with the run's last value; then copied back.
template <typename Float> void COO<Float>::sort(bool merge) {
  const size_t n = val.size();
  if (n == 0) return;
  void *d_r = internal::dalloc(sizeof(int) * n);
  void *d_c = internal::dalloc(sizeof(int) * n);
  void *d_v = internal::dalloc(sizeof(Float) * n);
  int64_t kept = 0;
  try {
    internal::h2d(d_r, row_index.data(), sizeof(int) * n);
    internal::h2d(d_c, col_index.data(), sizeof(int) * n);
    internal::h2d(d_v, val.data(), sizeof(Float) * n);
    internal::check(mlsh_coo_sort(internal::handle(), (int)rowN, (int)colN, (int64_t)n,
                                  static_cast<int *>(d_r), static_cast<int *>(d_c), d_v,
                                  internal::dtype<Float>(), merge ? 1 : 0, &kept),
                    "COO::sort");
    row_index.resize((size_t)kept);
    col_index.resize((size_t)kept);
    val.resize((size_t)kept);
    internal::d2h(row_index.data(), d_r, sizeof(int) * (size_t)kept);
    internal::d2h(col_index.data(), d_c, sizeof(int) * (size_t)kept);
    internal::d2h(val.data(), d_v, sizeof(Float) * (size_t)kept);
  } catch (...) {
    internal::dfree(d_r);
    internal::dfree(d_c);
    internal::dfree(d_v);
    throw;
  }
  internal::dfree(d_r);
  internal::dfree(d_c);
  internal::dfree(d_v);
}

template class COO<double>;
template class COO<float>;

// CRS from COO (src/utils/convert/convert_crs.cpp:9-43): entries must be
// ordered by row (a COO that is not gets sorted first); within a row their
// order is kept.  The row pointer is computed on the device.
template <typename Float> void CRS<Float>::convert(COO<Float> &coo) {
  rowN = coo.get_row();
  colN = coo.get_col();
  const size_t n = coo.get_nnz();
  for (size_t k = 1; k < n; ++k)
    if (coo.row_index[k] < coo.row_index[k - 1]) {
      coo.sort(false);
      break;
    }
  row_ptr.assign(rowN + 1, 0);
  col_ind.assign(coo.col_index.begin(), coo.col_index.end());
  alloc_val(n);
  std::copy(coo.val.begin(), coo.val.end(), val.get());
  void *d_r = internal::dalloc(sizeof(int) * std::max<size_t>(n, 1));
  void *d_p = internal::dalloc(sizeof(int) * (rowN + 1));
  try {
    if (n) internal::h2d(d_r, coo.row_index.data(), sizeof(int) * n);
    internal::check(mlsh_coo_to_csr(internal::handle(), (int)rowN, (int64_t)n,
                                    static_cast<const int *>(d_r), static_cast<int *>(d_p)),
                    "CRS::convert");
    internal::d2h(row_ptr.data(), d_p, sizeof(int) * (rowN + 1));
  } catch (...) {
    internal::dfree(d_r);
    internal::dfree(d_p);
    throw;
  }
  internal::dfree(d_r);
  internal::dfree(d_p);
  gpu_status = std::make_shared<bool>(false);
  dev.reset();
}
template void CRS<double>::convert(COO<double> &);
template void CRS<float>::convert(COO<float> &);

}  // namespace matrix

// ==================================================================== BLAS
namespace {
template <typename T> void need_device(const T &x, const char *what) {
  if (!x.get_device_mem_stat())
    throw std::runtime_error(std::string("error, ") + what +
                             ": operands must be device resident (util::send)");
}
template <typename A, typename B> void need_size(const A &a, const B &b, const char *what) {
  if (a.size() != b.size()) throw std::runtime_error(std::string("error, ") + what + ": size");
}

template <typename T>
void matvec_t(double a, const matrix::CRS<T> &A, const vector<T> &x, double b, vector<T> &y) {
  need_device(A, "matvec");
  need_device(x, "matvec");
  need_device(y, "matvec");
  if (A.get_col() != x.size() || A.get_row() != y.size())
    throw std::runtime_error("error, matvec: size");
  internal::check(mlsh_spmv(internal::handle(), A.device_plan(), a, x.device_data(), b,
                            y.device_data()),
                  "matvec");
}

template <typename T>
void matvec_tr(const matrix::CRS<T> &A, const vector<T> &x, vector<T> &y) {
  need_device(A, "matvec_T");
  need_device(x, "matvec_T");
  need_device(y, "matvec_T");
  if (A.get_row() != x.size() || A.get_col() != y.size())
    throw std::runtime_error("error, matvec_T: size");
  internal::check(mlsh_spmv_transpose(internal::handle(), A.device_plan(), 1.0,
                                      x.device_data(), 0.0, y.device_data()),
                  "matvec_T");
}

template <typename T> T dot_t(const vector<T> &x, const vector<T> &y) {
  need_device(x, "dot");
  need_device(y, "dot");
  need_size(x, y, "dot");
  double r = 0.0;
  internal::check(mlsh_dot(internal::handle(), internal::dtype<T>(), (int64_t)x.size(),
                           x.device_data(), y.device_data(), &r),
                  "dot");
  return (T)r;
}

template <typename T> T nrm2_t(const vector<T> &x) {
  need_device(x, "nrm2");
  double r = 0.0;
  internal::check(mlsh_nrm2(internal::handle(), internal::dtype<T>(), (int64_t)x.size(),
                            x.device_data(), &r),
                  "nrm2");
  return (T)r;
}
}  // namespace

namespace blas {
void matvec_T(const matrix::CRS<double> &A, const vector<double> &x, vector<double> &y) {
  matvec_tr<double>(A, x, y);
}
void matvec_T(const matrix::CRS<float> &A, const vector<float> &x, vector<float> &y) {
  matvec_tr<float>(A, x, y);
}
void matvec(const matrix::CRS<double> &A, const vector<double> &x, vector<double> &y) {
  matvec_t<double>(1.0, A, x, 0.0, y);
}
void matvec(const matrix::CRS<float> &A, const vector<float> &x, vector<float> &y) {
  matvec_t<float>(1.0, A, x, 0.0, y);
}
void matvec(const double &a, const matrix::CRS<double> &A, const vector<double> &x,
            const double &b, vector<double> &y) {
  matvec_t<double>(a, A, x, b, y);
}
void matvec(const float &a, const matrix::CRS<float> &A, const vector<float> &x,
            const float &b, vector<float> &y) {
  matvec_t<float>(a, A, x, b, y);
}

double dot(const vector<double> &x, const vector<double> &y) { return dot_t(x, y); }
float dot(const vector<float> &x, const vector<float> &y) { return dot_t(x, y); }
void dot(const vector<double> &x, const vector<double> &y, double &ans) { ans = dot_t(x, y); }
void dot(const vector<float> &x, const vector<float> &y, float &ans) { ans = dot_t(x, y); }
double nrm2(const vector<double> &x) { return nrm2_t(x); }
float nrm2(const vector<float> &x) { return nrm2_t(x); }
void nrm2(const vector<double> &x, double &ans) { ans = nrm2_t(x); }
void nrm2(const vector<float> &x, float &ans) { ans = nrm2_t(x); }

#define MLSH_AXPY_LIKE(NAME, CALL)                                                    \
  void NAME(const double alpha, const vector<double> &x, vector<double> &y) {         \
    need_device(x, #NAME);                                                            \
    need_device(y, #NAME);                                                            \
    need_size(x, y, #NAME);                                                           \
    internal::check(CALL(internal::handle(), MLSH_F64, (int64_t)x.size(), alpha,     \
                         x.device_data(), y.device_data()),                           \
                    #NAME);                                                           \
  }                                                                                   \
  void NAME(const float alpha, const vector<float> &x, vector<float> &y) {            \
    need_device(x, #NAME);                                                            \
    need_device(y, #NAME);                                                            \
    need_size(x, y, #NAME);                                                           \
    internal::check(CALL(internal::handle(), MLSH_F32, (int64_t)x.size(), alpha,     \
                         x.device_data(), y.device_data()),                           \
                    #NAME);                                                           \
  }
MLSH_AXPY_LIKE(axpy, mlsh_axpy)
MLSH_AXPY_LIKE(xpay, mlsh_xpay)
#undef MLSH_AXPY_LIKE

template <typename T>
static void axpyz_t(double alpha, const vector<T> &x, const vector<T> &y, vector<T> &z) {
  need_device(x, "axpyz");
  need_device(y, "axpyz");
  need_device(z, "axpyz");
  need_size(x, y, "axpyz");
  need_size(x, z, "axpyz");
  internal::check(mlsh_axpyz(internal::handle(), internal::dtype<T>(), (int64_t)x.size(), alpha,
                             x.device_data(), y.device_data(), z.device_data()),
                  "axpyz");
}
void axpyz(const double alpha, const vector<double> &x, const vector<double> &y,
           vector<double> &z) {
  axpyz_t(alpha, x, y, z);
}
void axpyz(const float alpha, const vector<float> &x, const vector<float> &y,
           vector<float> &z) {
  axpyz_t(alpha, x, y, z);
}

template <typename T> static void copy_t(const vector<T> &x, vector<T> &y) {
  need_device(x, "copy");
  need_device(y, "copy");
  need_size(x, y, "copy");
  internal::check(mlsh_copy(internal::handle(), internal::dtype<T>(), (int64_t)x.size(),
                            x.device_data(), y.device_data()),
                  "copy");
}
void copy(const vector<double> &x, vector<double> &y) { copy_t(x, y); }
void copy(const vector<float> &x, vector<float> &y) { copy_t(x, y); }
}  // namespace blas

// ===================================================================== VML
namespace vml {
template <typename T>
static void binop(int (*fn)(mlsh_handle, int, int64_t, const void *, const void *, void *),
                  const vector<T> &a, const vector<T> &b, vector<T> &y, const char *what) {
  need_device(a, what);
  need_device(b, what);
  need_device(y, what);
  need_size(a, b, what);
  need_size(a, y, what);
  internal::check(fn(internal::handle(), internal::dtype<T>(), (int64_t)a.size(),
                     a.device_data(), b.device_data(), y.device_data()),
                  what);
}
void sub(const vector<double> &a, const vector<double> &b, vector<double> &y) {
  binop(mlsh_vsub, a, b, y, "vml::sub");
}
void sub(const vector<float> &a, const vector<float> &b, vector<float> &y) {
  binop(mlsh_vsub, a, b, y, "vml::sub");
}
void mul(const vector<double> &a, const vector<double> &b, vector<double> &y) {
  binop(mlsh_vmul, a, b, y, "vml::mul");
}
void mul(const vector<float> &a, const vector<float> &b, vector<float> &y) {
  binop(mlsh_vmul, a, b, y, "vml::mul");
}
template <typename T> static void recip_t(const vector<T> &a, vector<T> &y) {
  need_device(a, "vml::reciprocal");
  need_device(y, "vml::reciprocal");
  need_size(a, y, "vml::reciprocal");
  internal::check(mlsh_vreciprocal(internal::handle(), internal::dtype<T>(), (int64_t)a.size(),
                                   a.device_data(), y.device_data()),
                  "vml::reciprocal");
}
void reciprocal(const vector<double> &a, vector<double> &y) { recip_t(a, y); }
void reciprocal(const vector<float> &a, vector<float> &y) { recip_t(a, y); }
}  // namespace vml

}  // namespace monolish
