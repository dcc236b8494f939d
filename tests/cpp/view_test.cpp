// view1D windows as BLAS / VML / matvec operands, written against the
// monolish API: every result is checked against the same arithmetic on the
// host, elements outside the windows must stay untouched, and a window of a
// window addresses the right slice.  Prints PASS when every check holds.
#include <cmath>
#include <iostream>
#include <vector>

#include "monolish_blas.hpp"
#include "monolish_vml.hpp"

namespace {

bool near(double a, double b, double tol) {
  return std::fabs(a - b) <= tol * std::max(1.0, std::fabs(b));
}

template <typename T> bool run(double tol) {
  using namespace monolish;
  bool ok = true;
  const size_t n = 1000, off = 123, len = 500;
  vector<T> x(n, -1.0, 1.0, 7u), y(n, -1.0, 1.0, 8u), z(n, 0.0);
  std::vector<double> hx(x.begin(), x.end()), hy(y.begin(), y.end());
  util::send(x, y, z);
  view1D<vector<T>, T> vx(x, off, len), vy(y, off + 10, len), vz(z, 300, len);

  // dot / nrm2 over windows
  double d = 0.0, s = 0.0;
  for (size_t i = 0; i < len; ++i) {
    d += hx[off + i] * hy[off + 10 + i];
    s += hx[off + i] * hx[off + i];
  }
  ok &= near((double)blas::dot(vx, vy), d, tol);
  ok &= near((double)blas::nrm2(vx), std::sqrt(s), tol);
  // a view and a vector of different sizes are rejected, as the reference does
  bool threw = false;
  try {
    T dd;
    blas::dot(vx, y, dd);
  } catch (const std::runtime_error &) {
    threw = true;
  }
  ok &= threw;

  // axpyz into a window of z: the rest of z stays 0
  blas::axpyz((T)0.5, vx, vy, vz);
  z.nonfree_recv();
  for (size_t i = 0; i < n; ++i) {
    const double want = (i >= 300 && i < 300 + len)
                            ? 0.5 * hx[off + i - 300] + hy[off + 10 + i - 300]
                            : 0.0;
    ok &= near((double)z.data()[i], want, tol);
  }

  // a window of a window, and vml on views
  view1D<vector<T>, T> vzz(vz, 100, 200);  // z[400, 600)
  view1D<vector<T>, T> vxx(vx, 100, 200);  // x[223, 423)
  vml::mul(vxx, vxx, vzz);
  z.nonfree_recv();
  for (size_t i = 0; i < 200; ++i)
    ok &= near((double)z.data()[400 + i], hx[223 + i] * hx[223 + i], tol);

  // matvec into a window: 2D Laplacian on 20x10, y window of a longer vector
  auto coo = util::laplacian_matrix_2D_5p<T>(20, 10);
  matrix::CRS<T> A(coo);
  vector<T> big(A.get_row() + 50, 0.0), src(A.get_row() + 7, -1.0, 1.0, 9u);
  std::vector<double> hs(src.begin(), src.end());
  util::send(A, big, src);
  view1D<vector<T>, T> vin(src, 7, A.get_row()), vout(big, 25, A.get_row());
  blas::matvec(A, vin, vout);
  big.nonfree_recv();
  for (size_t r = 0; r < A.get_row(); ++r) {
    double want = 0.0;
    for (int j = A.row_ptr[r]; j < A.row_ptr[r + 1]; ++j)
      want += (double)A.data()[j] * hs[7 + (size_t)A.col_ind[j]];
    ok &= near((double)big.data()[25 + r], want, tol * 10);
  }
  ok &= big.data()[24] == (T)0 && big.data()[25 + A.get_row()] == (T)0;

  // copy between windows and xpay on a window
  blas::copy(vx, vz);
  blas::xpay((T)2.0, vx, vz);  // vz = vx + 2 vz = 3 vx
  z.nonfree_recv();
  for (size_t i = 0; i < len; ++i) ok &= near((double)z.data()[300 + i], 3.0 * hx[off + i], tol);
  return ok;
}

}  // namespace

int main() {
  bool ok = run<double>(1e-12) && run<float>(1e-5);
  std::cout << (ok ? "PASS" : "FAIL") << std::endl;
  return ok ? 0 : 1;
}
