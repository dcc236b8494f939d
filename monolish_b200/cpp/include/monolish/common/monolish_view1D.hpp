// view1D over a vector: a window [first, first + size) of a monolish::vector
// (or of another such window), usable wherever the solve path's BLAS / VML
// take a vector (include/monolish/common/monolish_view1D.hpp of the
// reference, vector-backed views; Dense- and tensor-backed views are not
// part of this layer).  A view owns nothing: it shares its vector's host
// and device storage and residency, so the device operations run on the
// window's slice of the vector's device copy.
#pragma once
#include <type_traits>

#include "monolish/common/monolish_common.hpp"

namespace monolish {

template <typename TYPE, typename Float> class view1D;

template <typename Float> class view1D<vector<Float>, Float> {
 private:
  vector<Float> &target;
  size_t first;
  size_t range;

  void check_range() const {
    if (first + range > target.size())
      throw std::runtime_error("error, view1D: window exceeds the vector");
  }

 public:
  using value_type = Float;

  view1D(vector<Float> &x, const size_t start, const size_t size)
      : target(x), first(start), range(size) {
    check_range();
  }
  // a window of a window: offsets add up, the vector is shared
  view1D(view1D<vector<Float>, Float> &x, const size_t start, const size_t size)
      : target(x.get_target()), first(x.get_first() + start), range(size) {
    check_range();
  }

  [[nodiscard]] std::string type() const { return "view1D(vector)"; }
  [[nodiscard]] vector<Float> &get_target() const { return target; }

  // residency is the vector's
  void send() const { target.send(); }
  void recv() { target.recv(); }
  void nonfree_recv() { target.nonfree_recv(); }
  void device_free() const { target.device_free(); }
  [[nodiscard]] bool get_device_mem_stat() const { return target.get_device_mem_stat(); }

  [[nodiscard]] size_t size() const { return range; }
  [[nodiscard]] size_t get_nnz() const { return range; }
  [[nodiscard]] size_t get_first() const { return first; }
  [[nodiscard]] size_t get_last() const { return first + range; }
  [[nodiscard]] size_t get_offset() const { return first; }
  void set_first(size_t i) {
    first = i;
    check_range();
  }
  void set_last(size_t i) {
    if (i < first) throw std::runtime_error("error, view1D: last before first");
    range = i - first;
    check_range();
  }

  // host storage: data() is the vector's base, begin() the window's start
  [[nodiscard]] Float *data() const { return const_cast<Float *>(target.data()); }
  [[nodiscard]] Float *begin() const { return data() + first; }
  [[nodiscard]] Float *end() const { return begin() + range; }
  // device pointer of the window's first element (nullptr when not on the device)
  [[nodiscard]] Float *device_data() const {
    Float *d = target.device_data();
    return d ? d + first : nullptr;
  }

  [[nodiscard]] Float &operator[](const size_t i) const {
    if (get_device_mem_stat()) throw std::runtime_error("Error, GPU vector cant use operator[]");
    return data()[first + i];
  }

  void fill(Float value) {
    if (get_device_mem_stat()) {
      internal::check(mlsh_fill(internal::handle(), internal::dtype<Float>(),
                                static_cast<int64_t>(range), value, device_data()),
                      "view1D::fill");
    } else {
      for (size_t i = 0; i < range; ++i) begin()[i] = value;
    }
  }
};

namespace internal {
// Operand traits of the solve path's vector arguments.
template <class V> struct vec_traits { static constexpr bool ok = false; };
template <class F> struct vec_traits<vector<F>> {
  static constexpr bool ok = true;
  static constexpr bool view = false;
  using type = F;
};
template <class F> struct vec_traits<view1D<vector<F>, F>> {
  static constexpr bool ok = true;
  static constexpr bool view = true;
  using type = F;
};
template <class... V> constexpr bool vecs_v = (vec_traits<std::decay_t<V>>::ok && ...);
template <class... V> constexpr bool any_view_v = (vec_traits<std::decay_t<V>>::view || ...);
template <class A, class... V>
constexpr bool same_elem_v =
    (std::is_same_v<typename vec_traits<std::decay_t<A>>::type,
                    typename vec_traits<std::decay_t<V>>::type> && ...);
// Overloads for argument lists that hold at least one view (the plain
// vector ones are the non-template functions).
template <class... V>
using if_views_t =
    std::enable_if_t<vecs_v<V...> && any_view_v<V...> && same_elem_v<V...>, int>;
template <class V> using elem_t = typename vec_traits<std::decay_t<V>>::type;

template <class V> void need_device_vec(const V &x, const char *what) {
  if (!x.get_device_mem_stat())
    throw std::runtime_error(std::string("error, ") + what +
                             ": operands must be device resident (util::send)");
}
template <class A, class B> void need_same_size(const A &a, const B &b, const char *what) {
  if (a.size() != b.size()) throw std::runtime_error(std::string("error, ") + what + ": size");
}
}  // namespace internal

}  // namespace monolish
