// monolish-compatible BLAS for the sparse solve path (device-resident
// operands; every call runs an sm_100a kernel through include/mlsh.h).
//
//   matvec  include/monolish/blas/monolish_matvec_blas.hpp:3972 (CRS x vector),
//           alpha/beta overload src/blas/matrix/matvec/matvec_blas.cpp:3853
//   matvec_T (CRS^T x vector)
//   dot, nrm2, axpy, xpay, axpyz, copy
//           include/monolish/blas/monolish_vector_blas.hpp
#pragma once
#include "monolish/common/monolish_common.hpp"
#include "monolish/common/monolish_view1D.hpp"

namespace monolish {
namespace blas {

void matvec(const matrix::CRS<double> &A, const vector<double> &x, vector<double> &y);
void matvec(const matrix::CRS<float> &A, const vector<float> &x, vector<float> &y);
void matvec(const double &a, const matrix::CRS<double> &A, const vector<double> &x,
            const double &b, vector<double> &y);
void matvec(const float &a, const matrix::CRS<float> &A, const vector<float> &x,
            const float &b, vector<float> &y);

// y = A^T x  (include/monolish/blas/monolish_matvec_blas.hpp:4283,
// src/blas/matrix/matvec/crs_matvec.hpp:88-98)
void matvec_T(const matrix::CRS<double> &A, const vector<double> &x, vector<double> &y);
void matvec_T(const matrix::CRS<float> &A, const vector<float> &x, vector<float> &y);

double dot(const vector<double> &x, const vector<double> &y);
float dot(const vector<float> &x, const vector<float> &y);
void dot(const vector<double> &x, const vector<double> &y, double &ans);
void dot(const vector<float> &x, const vector<float> &y, float &ans);

double nrm2(const vector<double> &x);
float nrm2(const vector<float> &x);
void nrm2(const vector<double> &x, double &ans);
void nrm2(const vector<float> &x, float &ans);

void axpy(const double alpha, const vector<double> &x, vector<double> &y);
void axpy(const float alpha, const vector<float> &x, vector<float> &y);
void xpay(const double alpha, const vector<double> &x, vector<double> &y);
void xpay(const float alpha, const vector<float> &x, vector<float> &y);
void axpyz(const double alpha, const vector<double> &x, const vector<double> &y,
           vector<double> &z);
void axpyz(const float alpha, const vector<float> &x, const vector<float> &y,
           vector<float> &z);
void copy(const vector<double> &x, vector<double> &y);
void copy(const vector<float> &x, vector<float> &y);

// ------------------------------------------------- view1D operands --------
// The same operations when any vector argument is a view1D window
// (include/monolish/blas/monolish_vector_blas.hpp, view1D overloads).
template <class X, class Y, internal::if_views_t<X, Y> = 0>
internal::elem_t<X> dot(const X &x, const Y &y) {
  internal::need_device_vec(x, "dot");
  internal::need_device_vec(y, "dot");
  internal::need_same_size(x, y, "dot");
  double r = 0.0;
  internal::check(mlsh_dot(internal::handle(), internal::dtype<internal::elem_t<X>>(),
                           (int64_t)x.size(), x.device_data(), y.device_data(), &r),
                  "dot");
  return (internal::elem_t<X>)r;
}
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void dot(const X &x, const Y &y, internal::elem_t<X> &ans) {
  ans = dot(x, y);
}
template <class X, internal::if_views_t<X> = 0>
internal::elem_t<X> nrm2(const X &x) {
  internal::need_device_vec(x, "nrm2");
  double r = 0.0;
  internal::check(mlsh_nrm2(internal::handle(), internal::dtype<internal::elem_t<X>>(),
                            (int64_t)x.size(), x.device_data(), &r),
                  "nrm2");
  return (internal::elem_t<X>)r;
}
template <class X, internal::if_views_t<X> = 0>
void nrm2(const X &x, internal::elem_t<X> &ans) {
  ans = nrm2(x);
}
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void axpy(const internal::elem_t<X> alpha, const X &x, Y &y) {
  internal::need_device_vec(x, "axpy");
  internal::need_device_vec(y, "axpy");
  internal::need_same_size(x, y, "axpy");
  internal::check(mlsh_axpy(internal::handle(), internal::dtype<internal::elem_t<X>>(),
                            (int64_t)x.size(), alpha, x.device_data(), y.device_data()),
                  "axpy");
}
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void xpay(const internal::elem_t<X> alpha, const X &x, Y &y) {
  internal::need_device_vec(x, "xpay");
  internal::need_device_vec(y, "xpay");
  internal::need_same_size(x, y, "xpay");
  internal::check(mlsh_xpay(internal::handle(), internal::dtype<internal::elem_t<X>>(),
                            (int64_t)x.size(), alpha, x.device_data(), y.device_data()),
                  "xpay");
}
template <class X, class Y, class Z, internal::if_views_t<X, Y, Z> = 0>
void axpyz(const internal::elem_t<X> alpha, const X &x, const Y &y, Z &z) {
  internal::need_device_vec(x, "axpyz");
  internal::need_device_vec(y, "axpyz");
  internal::need_device_vec(z, "axpyz");
  internal::need_same_size(x, y, "axpyz");
  internal::need_same_size(x, z, "axpyz");
  internal::check(mlsh_axpyz(internal::handle(), internal::dtype<internal::elem_t<X>>(),
                             (int64_t)x.size(), alpha, x.device_data(), y.device_data(),
                             z.device_data()),
                  "axpyz");
}
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void copy(const X &x, Y &y) {
  internal::need_device_vec(x, "copy");
  internal::need_device_vec(y, "copy");
  internal::need_same_size(x, y, "copy");
  internal::check(mlsh_copy(internal::handle(), internal::dtype<internal::elem_t<X>>(),
                            (int64_t)x.size(), x.device_data(), y.device_data()),
                  "copy");
}
// y = A x and y = a A x + b y with view operands
// (include/monolish/blas/monolish_matvec_blas.hpp, view1D overloads)
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void matvec(const internal::elem_t<X> &a, const matrix::CRS<internal::elem_t<X>> &A, const X &x,
            const internal::elem_t<X> &b, Y &y) {
  internal::need_device_vec(x, "matvec");
  internal::need_device_vec(y, "matvec");
  if (!A.get_device_mem_stat())
    throw std::runtime_error("error, matvec: operands must be device resident (util::send)");
  if (A.get_col() != x.size() || A.get_row() != y.size())
    throw std::runtime_error("error, matvec: size");
  internal::check(mlsh_spmv(internal::handle(), A.device_plan(), a, x.device_data(), b,
                            y.device_data()),
                  "matvec");
}
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void matvec(const matrix::CRS<internal::elem_t<X>> &A, const X &x, Y &y) {
  matvec((internal::elem_t<X>)1, A, x, (internal::elem_t<X>)0, y);
}
template <class X, class Y, internal::if_views_t<X, Y> = 0>
void matvec_T(const matrix::CRS<internal::elem_t<X>> &A, const X &x, Y &y) {
  internal::need_device_vec(x, "matvec_T");
  internal::need_device_vec(y, "matvec_T");
  if (!A.get_device_mem_stat())
    throw std::runtime_error("error, matvec_T: operands must be device resident (util::send)");
  if (A.get_row() != x.size() || A.get_col() != y.size())
    throw std::runtime_error("error, matvec_T: size");
  internal::check(mlsh_spmv_transpose(internal::handle(), A.device_plan(), 1.0,
                                      x.device_data(), 0.0, y.device_data()),
                  "matvec_T");
}

}  // namespace blas
}  // namespace monolish
