// monolish-compatible containers over the B200 C ABI (include/mlsh.h).
//
// Drop-in for the parts of monolish's container API that the sparse solve
// path uses:
//   vector<T>          include/monolish/common/monolish_vector.hpp:47-764
//   matrix::COO<T>     include/monolish/common/monolish_coo.hpp (host-side
//                      construction and MatrixMarket input only)
//   matrix::CRS<T>     include/monolish/common/monolish_crs.hpp:39-859
//   util::send/recv/device_free/nonfree_recv   monolish_common.hpp:1174-1223
//   solver status codes                         monolish_common.hpp:16-21
//
// Residency follows the reference: containers own host arrays; send()
// copies them to the device (allocating on first use) and marks the object
// device-resident; recv() copies back and frees the device copy;
// nonfree_recv() copies back and keeps it; device_free() drops it.
// Computation (blas::, vml::, equation::) runs only on device-resident
// operands: the GPU kernels are the implementation, and a host-resident
// operand is an error (std::runtime_error), never a silent CPU path.
#pragma once

#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <iostream>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlsh.h"

#define MONOLISH_SOLVER_SUCCESS 0
#define MONOLISH_SOLVER_SIZE_ERROR -1
#define MONOLISH_SOLVER_MAXITER -2
#define MONOLISH_SOLVER_BREAKDOWN -3
#define MONOLISH_SOLVER_RESIDUAL_NAN -4
#define MONOLISH_SOLVER_NOT_IMPL -10

namespace monolish {

namespace internal {
// Per-thread handle on the current device (created on first use).
mlsh_handle handle();
// Throws std::runtime_error for library errors (status < -9).
void check(int status, const char *what);
void *dalloc(size_t bytes);
void dfree(void *p);
void h2d(void *d, const void *h, size_t bytes);
void d2h(void *h, const void *d, size_t bytes);
void d2d(void *d, const void *s, size_t bytes);
template <typename T> constexpr int dtype() { return sizeof(T) == 8 ? MLSH_F64 : MLSH_F32; }

// Device buffer with shared ownership.
template <typename T> std::shared_ptr<T> dshared(size_t n) {
  T *p = n ? static_cast<T *>(dalloc(sizeof(T) * n)) : nullptr;
  return std::shared_ptr<T>(p, [](T *q) { dfree(q); });
}
}  // namespace internal

namespace util {
// Logger controls (monolish_common.hpp, logger_utils.cpp).  Level >= 1
// writes one YAML-like line per solver call to the log file (stdout if no
// file); nothing synchronises inside an iteration.
void set_log_level(size_t level);
void set_log_filename(std::string filename);
bool build_with_gpu();
}  // namespace util

// ------------------------------------------------------------------ vector
template <typename Float> class vector {
 private:
  size_t n_ = 0;
  std::shared_ptr<Float> val;
  mutable std::shared_ptr<Float> dval;
  mutable std::shared_ptr<bool> gpu_status = std::make_shared<bool>(false);

  void alloc(size_t N) {
    n_ = N;
    val = std::shared_ptr<Float>(new Float[N > 0 ? N : 1], std::default_delete<Float[]>());
  }

 public:
  vector() { alloc(0); }
  explicit vector(const size_t N) {
    alloc(N);
    for (size_t i = 0; i < N; ++i) val.get()[i] = Float(0);
  }
  vector(const size_t N, const Float value) {
    alloc(N);
    for (size_t i = 0; i < N; ++i) val.get()[i] = value;
  }
  vector(const std::vector<Float> &v) {
    alloc(v.size());
    for (size_t i = 0; i < n_; ++i) val.get()[i] = v[i];
  }
  vector(const std::initializer_list<Float> &list) {
    alloc(list.size());
    size_t i = 0;
    for (auto x : list) val.get()[i++] = x;
  }
  vector(const Float *start, const Float *end) {
    alloc(static_cast<size_t>(end - start));
    for (size_t i = 0; i < n_; ++i) val.get()[i] = start[i];
  }
  // random vector from std::random_device (vector_constructor.cpp:54-70)
  vector(const size_t N, const Float min, const Float max) {
    alloc(N);
    std::random_device rd;
    std::mt19937 mt(rd());
    std::uniform_real_distribution<> rand(min, max);
    for (size_t i = 0; i < N; ++i) val.get()[i] = rand(mt);
  }
  // seeded random vector (vector_constructor.cpp:98-110): mt19937(seed)
  // with uniform_real_distribution<double>, identical values
  vector(const size_t N, const Float min, const Float max, const std::uint32_t seed) {
    alloc(N);
    std::mt19937 mt(seed);
    std::uniform_real_distribution<> rand(min, max);
    for (size_t i = 0; i < N; ++i) val.get()[i] = rand(mt);
  }
  // copy: host data always; device data too when the source is on the device
  vector(const vector<Float> &v) {
    alloc(v.n_);
    for (size_t i = 0; i < n_; ++i) val.get()[i] = v.val.get()[i];
    if (v.get_device_mem_stat()) {
      dval = internal::dshared<Float>(n_);
      internal::d2d(dval.get(), v.dval.get(), sizeof(Float) * n_);
      *gpu_status = true;
    }
  }
  vector<Float> &operator=(const vector<Float> &v) {
    if (this == &v) return *this;
    if (get_device_mem_stat()) {
      if (!v.get_device_mem_stat() || v.n_ != n_)
        throw std::runtime_error("error, vector operator=: device status or size mismatch");
      internal::d2d(dval.get(), v.dval.get(), sizeof(Float) * n_);
      return *this;
    }
    alloc(v.n_);
    for (size_t i = 0; i < n_; ++i) val.get()[i] = v.val.get()[i];
    if (v.get_device_mem_stat()) {
      dval = internal::dshared<Float>(n_);
      internal::d2d(dval.get(), v.dval.get(), sizeof(Float) * n_);
      *gpu_status = true;
    }
    return *this;
  }

  // ------------------------------------------------------------ residency
  void send() const {
    if (!dval && n_ > 0) dval = internal::dshared<Float>(n_);
    internal::h2d(dval.get(), val.get(), sizeof(Float) * n_);
    *gpu_status = true;
  }
  void recv() {
    nonfree_recv();
    device_free();
  }
  void nonfree_recv() {
    if (get_device_mem_stat()) internal::d2h(val.get(), dval.get(), sizeof(Float) * n_);
  }
  void device_free() const {
    dval.reset();
    *gpu_status = false;
  }
  [[nodiscard]] bool get_device_mem_stat() const { return *gpu_status; }

  // ------------------------------------------------------------- access
  [[nodiscard]] size_t size() const { return n_; }
  [[nodiscard]] size_t get_nnz() const { return n_; }
  [[nodiscard]] Float *data() { return val.get(); }
  [[nodiscard]] const Float *data() const { return val.get(); }
  [[nodiscard]] Float *begin() { return val.get(); }
  [[nodiscard]] const Float *begin() const { return val.get(); }
  [[nodiscard]] Float *end() { return val.get() + n_; }
  [[nodiscard]] const Float *end() const { return val.get() + n_; }
  // device pointer (extension; nullptr when not on the device)
  [[nodiscard]] Float *device_data() const { return dval.get(); }
  [[nodiscard]] Float &operator[](size_t i) {
    if (get_device_mem_stat()) throw std::runtime_error("Error, GPU vector cant use operator[]");
    return val.get()[i];
  }
  [[nodiscard]] const Float &operator[](size_t i) const {
    if (get_device_mem_stat()) throw std::runtime_error("Error, GPU vector cant use operator[]");
    return val.get()[i];
  }
  void fill(Float value) {
    if (get_device_mem_stat()) {
      internal::check(mlsh_fill(internal::handle(), internal::dtype<Float>(),
                                static_cast<int64_t>(n_), value, dval.get()),
                      "vector::fill");
    } else {
      for (size_t i = 0; i < n_; ++i) val.get()[i] = value;
    }
  }
  void resize(size_t N, Float v = 0) {
    if (get_device_mem_stat()) throw std::runtime_error("Error, GPU vector cant use resize");
    std::shared_ptr<Float> old = val;
    const size_t m = n_;
    alloc(N);
    for (size_t i = 0; i < N; ++i) val.get()[i] = i < m ? old.get()[i] : v;
  }
  void print_all(bool force_cpu = false) const {
    (void)force_cpu;
    if (get_device_mem_stat()) {
      std::vector<Float> tmp(n_);
      internal::d2h(tmp.data(), dval.get(), sizeof(Float) * n_);
      for (auto x : tmp) std::cout << x << std::endl;
    } else {
      for (size_t i = 0; i < n_; ++i) std::cout << val.get()[i] << std::endl;
    }
  }
};

namespace matrix {

// ------------------------------------------------------------------- COO
// Host-side coordinate matrix used to build CRS (construction and
// MatrixMarket input; src/utils/IO/IO_coo.cpp:69-153 and
// src/utils/convert/convert_crs.cpp:9-43 for the CRS conversion).
template <typename Float> class COO {
 public:
  std::vector<int> row_index;
  std::vector<int> col_index;
  std::vector<Float> val;
  COO() = default;
  COO(const size_t M, const size_t N) : rowN(M), colN(N) {}
  explicit COO(const std::string filename) { input_mm(filename); }
  COO(const size_t M, const size_t N, const size_t NNZ, const int *row, const int *col,
      const Float *value)
      : row_index(row, row + NNZ), col_index(col, col + NNZ), val(value, value + NNZ),
        rowN(M), colN(N) {}
  void input_mm(const std::string filename);
  void insert(const size_t m, const size_t n, const Float value) {
    row_index.push_back(static_cast<int>(m));
    col_index.push_back(static_cast<int>(n));
    val.push_back(value);
  }
  // sort by (row, col), equal (row, col) in input order; with merge each
  // run of equal (row, col) becomes one entry holding the run's last value
  void sort(bool merge);
  [[nodiscard]] size_t get_row() const { return rowN; }
  [[nodiscard]] size_t get_col() const { return colN; }
  [[nodiscard]] size_t get_nnz() const { return val.size(); }

 private:
  size_t rowN = 0, colN = 0;
};

// ------------------------------------------------------------------- CRS
template <typename Float> class CRS {
 public:
  std::vector<int> row_ptr;
  std::vector<int> col_ind;

 private:
  size_t rowN = 0, colN = 0, nnz = 0;
  std::shared_ptr<Float> val;
  // device copies and the SpMV plan, shared between copies of the object
  struct Device {
    std::shared_ptr<int> rp, ci;
    std::shared_ptr<Float> v;
    mlsh_csr_plan plan = nullptr;
    ~Device() {
      if (plan) mlsh_csr_plan_destroy(plan);
    }
  };
  mutable std::shared_ptr<Device> dev;
  mutable std::shared_ptr<bool> gpu_status = std::make_shared<bool>(false);

  void alloc_val(size_t NNZ) {
    nnz = NNZ;
    val = std::shared_ptr<Float>(new Float[NNZ > 0 ? NNZ : 1], std::default_delete<Float[]>());
  }

 public:
  CRS() { alloc_val(0); row_ptr.assign(1, 0); }
  CRS(const size_t M, const size_t N, const size_t NNZ) : rowN(M), colN(N) {
    row_ptr.assign(M + 1, 0);
    col_ind.assign(NNZ, 0);
    alloc_val(NNZ);
  }
  CRS(const size_t M, const size_t N, const size_t NNZ, const int *rowptr, const int *colind,
      const Float *value)
      : row_ptr(rowptr, rowptr + M + 1), col_ind(colind, colind + NNZ), rowN(M), colN(N) {
    alloc_val(NNZ);
    for (size_t i = 0; i < NNZ; ++i) val.get()[i] = value[i];
  }
  CRS(const size_t M, const size_t N, const std::vector<int> &rowptr,
      const std::vector<int> &colind, const std::vector<Float> &value)
      : row_ptr(rowptr), col_ind(colind), rowN(M), colN(N) {
    alloc_val(value.size());
    for (size_t i = 0; i < nnz; ++i) val.get()[i] = value[i];
  }
  explicit CRS(COO<Float> &coo) { convert(coo); }
  CRS(const CRS<Float> &A)
      : row_ptr(A.row_ptr), col_ind(A.col_ind), rowN(A.rowN), colN(A.colN) {
    alloc_val(A.nnz);
    for (size_t i = 0; i < nnz; ++i) val.get()[i] = A.val.get()[i];
    if (A.get_device_mem_stat()) {
      send();
      internal::d2d(dev->v.get(), A.dev->v.get(), sizeof(Float) * nnz);
    }
  }
  ~CRS() = default;

  void convert(COO<Float> &coo);

  // ------------------------------------------------------------ residency
  void send() const {
    if (!dev) {
      dev = std::make_shared<Device>();
      dev->rp = internal::dshared<int>(rowN + 1);
      dev->ci = internal::dshared<int>(nnz);
      dev->v = internal::dshared<Float>(nnz);
    }
    internal::h2d(dev->rp.get(), row_ptr.data(), sizeof(int) * (rowN + 1));
    internal::h2d(dev->ci.get(), col_ind.data(), sizeof(int) * nnz);
    internal::h2d(dev->v.get(), val.get(), sizeof(Float) * nnz);
    if (dev->plan == nullptr) {
      internal::check(mlsh_csr_plan_create(internal::handle(), static_cast<int>(rowN),
                                           static_cast<int>(colN), static_cast<int>(nnz),
                                           dev->rp.get(), dev->ci.get(), dev->v.get(),
                                           internal::dtype<Float>(), row_ptr.data(), 1,
                                           &dev->plan),
                      "CRS::send");
    } else {
      internal::check(mlsh_csr_plan_values_changed(dev->plan), "CRS::send");
    }
    *gpu_status = true;
  }
  void recv() {
    nonfree_recv();
    device_free();
  }
  void nonfree_recv() {
    if (get_device_mem_stat())
      internal::d2h(val.get(), dev->v.get(), sizeof(Float) * nnz);
  }
  void device_free() const {
    dev.reset();
    *gpu_status = false;
  }
  [[nodiscard]] bool get_device_mem_stat() const { return *gpu_status; }

  // --------------------------------------------------------------- access
  [[nodiscard]] size_t get_row() const { return rowN; }
  [[nodiscard]] size_t get_col() const { return colN; }
  [[nodiscard]] size_t get_nnz() const { return nnz; }
  [[nodiscard]] std::string type() const { return "CRS"; }
  [[nodiscard]] Float *data() { return val.get(); }
  [[nodiscard]] const Float *data() const { return val.get(); }
  [[nodiscard]] Float *begin() { return val.get(); }
  [[nodiscard]] const Float *begin() const { return val.get(); }
  // the SpMV plan (extension; nullptr when not on the device)
  [[nodiscard]] mlsh_csr_plan device_plan() const { return dev ? dev->plan : nullptr; }

  // diagonal (src/utils/getvec/crs_getvec.cpp:8-55)
  void diag(vector<Float> &vec) const {
    if (!get_device_mem_stat() || !vec.get_device_mem_stat())
      throw std::runtime_error("error, CRS::diag needs device-resident operands");
    if (vec.size() < (rowN < colN ? rowN : colN))
      throw std::runtime_error("error, CRS::diag: vector too short");
    internal::check(mlsh_csr_diag(internal::handle(), dev->plan, vec.device_data()), "diag");
  }

  void print_all(bool force_cpu = false) const {
    (void)force_cpu;
    std::vector<Float> v(val.get(), val.get() + nnz);
    if (get_device_mem_stat()) internal::d2h(v.data(), dev->v.get(), sizeof(Float) * nnz);
    for (size_t i = 0; i < rowN; ++i)
      for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j)
        std::cout << i + 1 << " " << col_ind[j] + 1 << " " << v[j] << std::endl;
  }
};

}  // namespace matrix

namespace util {
template <typename T> void send(T &x) { x.send(); }
template <typename T, typename... Types> void send(T &x, Types &...args) {
  x.send();
  send(args...);
}
template <typename T> void recv(T &x) { x.recv(); }
template <typename T, typename... Types> void recv(T &x, Types &...args) {
  x.recv();
  recv(args...);
}
template <typename T> void nonfree_recv(T &x) { x.nonfree_recv(); }
template <typename T, typename... Types> void nonfree_recv(T &x, Types &...args) {
  x.nonfree_recv();
  nonfree_recv(args...);
}
template <typename T> void device_free(T &x) { x.device_free(); }
template <typename T, typename... Types> void device_free(T &x, Types &...args) {
  x.device_free();
  device_free(args...);
}

// Seeded random fill (src/utils/vector_constructor.cpp:72-96).
template <typename T>
void random_vector(vector<T> &vec, const T min, const T max, const std::uint32_t seed) {
  std::mt19937 mt(seed);
  std::uniform_real_distribution<> rand(min, max);
  for (size_t i = 0; i < vec.size(); ++i) vec[i] = rand(mt);
}

// 2D 5-point Laplacian as COO (src/utils/create_matrix/laplacian_2D5p.cpp).
template <typename T> matrix::COO<T> laplacian_matrix_2D_5p(const int m, const int n);

// solver_check: kept exactly as the reference behaves
// (src/utils/equation_utils.cpp:7-28): it returns false for every code, so
// callers detect failure only by checking the answer.
bool solver_check(const int err);
}  // namespace util

}  // namespace monolish
