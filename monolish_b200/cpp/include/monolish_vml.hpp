// monolish-compatible vector math used by the solve path
// (include/monolish/vml/monolish_vector_vml.hpp: sub, mul, reciprocal).
#pragma once
#include "monolish/common/monolish_common.hpp"
#include "monolish/common/monolish_view1D.hpp"

namespace monolish {
namespace vml {

void sub(const vector<double> &a, const vector<double> &b, vector<double> &y);
void sub(const vector<float> &a, const vector<float> &b, vector<float> &y);
void mul(const vector<double> &a, const vector<double> &b, vector<double> &y);
void mul(const vector<float> &a, const vector<float> &b, vector<float> &y);
void reciprocal(const vector<double> &a, vector<double> &y);
void reciprocal(const vector<float> &a, vector<float> &y);

// view1D operands (include/monolish/vml/monolish_vector_vml.hpp, view1D
// overloads)
template <class A, class B, class Y, internal::if_views_t<A, B, Y> = 0>
void sub(const A &a, const B &b, Y &y) {
  internal::need_device_vec(a, "sub");
  internal::need_device_vec(b, "sub");
  internal::need_device_vec(y, "sub");
  internal::need_same_size(a, b, "sub");
  internal::need_same_size(a, y, "sub");
  internal::check(mlsh_vsub(internal::handle(), internal::dtype<internal::elem_t<A>>(),
                            (int64_t)a.size(), a.device_data(), b.device_data(), y.device_data()),
                  "sub");
}
template <class A, class B, class Y, internal::if_views_t<A, B, Y> = 0>
void mul(const A &a, const B &b, Y &y) {
  internal::need_device_vec(a, "mul");
  internal::need_device_vec(b, "mul");
  internal::need_device_vec(y, "mul");
  internal::need_same_size(a, b, "mul");
  internal::need_same_size(a, y, "mul");
  internal::check(mlsh_vmul(internal::handle(), internal::dtype<internal::elem_t<A>>(),
                            (int64_t)a.size(), a.device_data(), b.device_data(), y.device_data()),
                  "mul");
}
template <class A, class Y, internal::if_views_t<A, Y> = 0>
void reciprocal(const A &a, Y &y) {
  internal::need_device_vec(a, "reciprocal");
  internal::need_device_vec(y, "reciprocal");
  internal::need_same_size(a, y, "reciprocal");
  internal::check(mlsh_vreciprocal(internal::handle(), internal::dtype<internal::elem_t<A>>(),
                                   (int64_t)a.size(), a.device_data(), y.device_data()),
                  "reciprocal");
}

}  // namespace vml
}  // namespace monolish
