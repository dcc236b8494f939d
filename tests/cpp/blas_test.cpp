// BLAS / VML test written against the monolish API and built against the
// B200 drop-in headers.  Each device result is compared with a plain host
// loop, with the reference test suite's tolerances (vector ops 1e-8 double /
// 1e-4 float; matvec 1e-6 / 1e-3, test/matrix/matrix_blas.cpp).
#include <cmath>
#include <iostream>
#include <vector>

#include "monolish_blas.hpp"
#include "monolish_equation.hpp"
#include "monolish_vml.hpp"

namespace {

bool near(double a, double b, double tol) {
  return std::fabs(a - b) <= tol * std::max(1.0, std::fabs(b));
}

template <typename T> bool check_vec(const char *what, const monolish::vector<T> &got,
                                     const std::vector<double> &want, double tol) {
  for (size_t i = 0; i < want.size(); ++i)
    if (!near(got.data()[i], want[i], tol)) {
      std::cout << what << " mismatch at " << i << ": " << got.data()[i] << " vs " << want[i]
                << std::endl;
      return false;
    }
  return true;
}

template <typename T> bool run(size_t n, double tol, double mv_tol) {
  using namespace monolish;
  bool ok = true;
  vector<T> x(n, -1.0, 1.0, 7u), y(n, -1.0, 1.0, 8u), z(n, 0.0);
  std::vector<double> hx(x.begin(), x.end()), hy(y.begin(), y.end());
  util::send(x, y, z);

  double d = 0.0, nn = 0.0;
  for (size_t i = 0; i < n; ++i) {
    d += hx[i] * hy[i];
    nn += hx[i] * hx[i];
  }
  ok &= near(blas::dot(x, y), d, tol);
  ok &= near(blas::nrm2(x), std::sqrt(nn), tol);

  const T a = (T)0.625;
  std::vector<double> w(n);
  vector<T> y2(y);  // device copy
  blas::axpy(a, x, y2);
  y2.nonfree_recv();
  for (size_t i = 0; i < n; ++i) w[i] = a * hx[i] + hy[i];
  ok &= check_vec("axpy", y2, w, tol);

  vector<T> y3(y);
  blas::xpay(a, x, y3);
  y3.nonfree_recv();
  for (size_t i = 0; i < n; ++i) w[i] = hx[i] + a * hy[i];
  ok &= check_vec("xpay", y3, w, tol);

  blas::axpyz(a, x, y, z);
  z.nonfree_recv();
  for (size_t i = 0; i < n; ++i) w[i] = a * hx[i] + hy[i];
  ok &= check_vec("axpyz", z, w, tol);

  vml::sub(x, y, z);
  z.nonfree_recv();
  for (size_t i = 0; i < n; ++i) w[i] = hx[i] - hy[i];
  ok &= check_vec("sub", z, w, tol);

  vml::mul(x, y, z);
  z.nonfree_recv();
  for (size_t i = 0; i < n; ++i) w[i] = hx[i] * hy[i];
  ok &= check_vec("mul", z, w, tol);

  blas::copy(x, z);
  z.nonfree_recv();
  ok &= check_vec("copy", z, hx, 0.0);

  // matvec on the 2D Laplacian built by util::laplacian_matrix_2D_5p
  auto coo = util::laplacian_matrix_2D_5p<T>(40, 30);
  matrix::CRS<T> A(coo);
  vector<T> v(A.get_row(), -1.0, 1.0, 9u), u(A.get_row(), 0.0);
  std::vector<double> hv(v.begin(), v.end()), mv(A.get_row(), 0.0);
  for (size_t i = 0; i < A.get_row(); ++i)
    for (int j = A.row_ptr[i]; j < A.row_ptr[i + 1]; ++j)
      mv[i] += (double)A.data()[j] * hv[(size_t)A.col_ind[j]];
  util::send(A, v, u);
  blas::matvec(A, v, u);
  u.recv();
  ok &= check_vec("matvec", u, mv, mv_tol);

  // COO -> CRS on the device from unsorted entries with one repeated
  // (row, col) (COO::sort keeps its last value), then matvec_T
  {
    const size_t m = 7, nc = 5;
    const std::vector<int> r = {3, 0, 6, 2, 0, 3, 5, 1, 4, 6};
    const std::vector<int> c = {1, 4, 0, 2, 1, 1, 3, 0, 4, 2};
    const std::vector<T> vals = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
    matrix::COO<T> C(m, nc, r.size(), r.data(), c.data(), vals.data());
    C.sort(true);
    ok &= C.get_nnz() == 9;
    for (size_t k = 1; k < C.get_nnz(); ++k)
      ok &= C.row_index[k - 1] < C.row_index[k] ||
            (C.row_index[k - 1] == C.row_index[k] && C.col_index[k - 1] < C.col_index[k]);
    std::vector<double> dense(m * nc, 0.0);
    for (size_t k = 0; k < r.size(); ++k) dense[(size_t)r[k] * nc + (size_t)c[k]] = vals[k];
    matrix::CRS<T> B(C);
    vector<T> xr(m, -1.0, 1.0, 3u), yr(nc, 0.0);
    std::vector<double> yt(nc, 0.0);
    for (size_t i = 0; i < m; ++i)
      for (size_t j = 0; j < nc; ++j) yt[j] += dense[i * nc + j] * (double)xr.data()[i];
    util::send(B, xr, yr);
    blas::matvec_T(B, xr, yr);
    yr.recv();
    ok &= check_vec("matvec_T", yr, yt, mv_tol);
  }

  // diag + Jacobi create/apply
  vector<T> dg(A.get_row(), 0.0);
  dg.send();
  A.diag(dg);
  dg.recv();
  for (size_t i = 0; i < A.get_row(); ++i) ok &= (dg.data()[i] == (T)4.0);

  // host-resident operands are rejected, not silently computed on the CPU
  vector<T> h1(4, 1.0), h2(4, 2.0);
  bool threw = false;
  try {
    (void)blas::dot(h1, h2);
  } catch (const std::runtime_error &) {
    threw = true;
  }
  ok &= threw;
  return ok;
}

}  // namespace

int main() {
  bool ok = run<double>(12345, 1e-8, 1e-6);
  ok &= run<float>(12345, 1e-4, 1e-3);
  std::cout << (ok ? "PASS" : "FAIL") << std::endl;
  return ok ? 0 : 1;
}
