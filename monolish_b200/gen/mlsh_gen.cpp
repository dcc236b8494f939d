// Seeded synthetic input generators (host C++).
//
// These build the workloads' CRS matrices and vectors bit-for-bit the same
// for every consumer (the CUDA library's tests and benchmarks, the CPU
// restatement and the reference CPU library).  They are setup code, not part
// of the solve path.
//
// Matrix families:
//   2D 5-point Laplacian  -- same row/column order and values as the
//       reference's util::laplacian_matrix_2D_5p
//       (src/utils/create_matrix/laplacian_2D5p.cpp:7-50): per row the
//       entries -m, -1, diag(4), +1, +m in ascending column order.
//   3D 7-point Laplacian  -- row ((k*m)+j)*m+i, diag 6, off-diagonals -1,
//       ascending columns, Dirichlet neighbours dropped.
//   Zipf(s) random rows   -- row length from a Zipf(s) law truncated to
//       [1, maxlen], columns uniform without replacement (Floyd's
//       algorithm) then sorted, values U[-1,1].  Each row draws from its own
//       splitmix64 stream keyed by (seed, row), so the matrix does not depend
//       on the thread count.
//   3D convection-diffusion -- first-order upwind 7-point stencil on an m^3
//       interior grid, h = 1/(m+1), diffusion D, velocity s*(1,0.5,0.25)
//       with s set by the cell Peclet number Pe = max|v_i|*h/(2D).
//   2D/3D variable-coefficient diffusion -- k = exp(N(0,1)) per cell,
//       harmonic face averaging 2 ka kb/(ka+kb); a Dirichlet face uses the
//       cell's own k (doubled-distance convention).
//
// Vectors: gen_uniform_mt reproduces the reference's seeded constructor
// vector(N, min, max, seed) (src/utils/vector_constructor.cpp:98-110):
// std::mt19937(seed) with std::uniform_real_distribution<double>.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  // uniform in [0, 1) with 53 random bits
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  // standard normal (Box-Muller)
  double normal() {
    double u1 = uniform();
    double u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

uint64_t stream_key(uint64_t seed, uint64_t idx) {
  SplitMix64 a(seed * 0x2545F4914F6CDD1DULL + 0x1234567ULL);
  uint64_t k = a.next();
  SplitMix64 b(k ^ (idx * 0x9E3779B97F4A7C15ULL));
  return b.next();
}

template <typename T>
void fill_uniform_mt(long n, double lo, double hi, unsigned seed, T *out) {
  std::mt19937 mt(seed);
  std::uniform_real_distribution<> rand(lo, hi);
  for (long i = 0; i < n; i++) out[i] = static_cast<T>(rand(mt));
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- vectors
void gen_uniform_mt_d(long n, double lo, double hi, unsigned seed, double *out) {
  fill_uniform_mt<double>(n, lo, hi, seed, out);
}
void gen_uniform_mt_s(long n, double lo, double hi, unsigned seed, float *out) {
  fill_uniform_mt<float>(n, lo, hi, seed, out);
}

// ------------------------------------------------------ 2D 5-point Poisson
long gen_lap2d5p_nnz(int m, int n) {
  long nn = (long)m * n;
  return 5 * nn - 2L * m - 2L * n;
}
// m = points per row of the grid (fast index), n = number of grid rows.
void gen_lap2d5p_fill(int m, int n, int *rp, int *ci, double *v) {
  int size = m * n;
  int k = 0;
  rp[0] = 0;
  for (int ii = 0; ii < size; ii++) {
    int i = ii / m;
    int j = ii - i * m;
    if (i > 0) { ci[k] = ii - m; v[k++] = -1.0; }
    if (j > 0) { ci[k] = ii - 1; v[k++] = -1.0; }
    ci[k] = ii; v[k++] = 4.0;
    if (j < m - 1) { ci[k] = ii + 1; v[k++] = -1.0; }
    if (i < n - 1) { ci[k] = ii + m; v[k++] = -1.0; }
    rp[ii + 1] = k;
  }
}

// ------------------------------------------------------ 3D 7-point Poisson
long gen_lap3d7p_nnz(int m) {
  long n = (long)m * m * m;
  return 7 * n - 6L * m * m;
}
void gen_lap3d7p_fill(int m, int *rp, int *ci, double *v) {
  const long n = (long)m * m * m;
  const long mm = (long)m * m;
  long pos = 0;
  rp[0] = 0;
  for (long r = 0; r < n; r++) {
    int i = (int)(r % m), j = (int)((r / m) % m), k = (int)(r / mm);
    pos += 1 + (i > 0) + (i < m - 1) + (j > 0) + (j < m - 1) + (k > 0) + (k < m - 1);
    rp[r + 1] = (int)pos;
  }
  #pragma omp parallel for schedule(static)
  for (long r = 0; r < n; r++) {
    int i = (int)(r % m), j = (int)((r / m) % m), k = (int)(r / mm);
    long q = rp[r];
    if (k > 0) { ci[q] = (int)(r - mm); v[q++] = -1.0; }
    if (j > 0) { ci[q] = (int)(r - m); v[q++] = -1.0; }
    if (i > 0) { ci[q] = (int)(r - 1); v[q++] = -1.0; }
    ci[q] = (int)r; v[q++] = 6.0;
    if (i < m - 1) { ci[q] = (int)(r + 1); v[q++] = -1.0; }
    if (j < m - 1) { ci[q] = (int)(r + m); v[q++] = -1.0; }
    if (k < m - 1) { ci[q] = (int)(r + mm); v[q++] = -1.0; }
  }
}

// ------------------------------------------------------------- Zipf rows
// Fills rp (n+1) from per-row Zipf(s) lengths in [1, maxlen] (each clamped to
// ncols); returns nnz (or -1 if it overflows int32).
long gen_zipf_rowptr(int n, int ncols, double s, int maxlen, uint64_t seed,
                     int *rp) {
  std::vector<double> cdf(maxlen);
  double acc = 0.0;
  for (int k = 1; k <= maxlen; k++) {
    acc += std::pow((double)k, -s);
    cdf[k - 1] = acc;
  }
  for (int k = 0; k < maxlen; k++) cdf[k] /= acc;
  std::vector<int> len(n);
  #pragma omp parallel for schedule(static)
  for (int r = 0; r < n; r++) {
    SplitMix64 g(stream_key(seed, (uint64_t)r));
    double u = g.uniform();
    int L = (int)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
    if (L > maxlen) L = maxlen;
    if (L > ncols) L = ncols;
    len[r] = L;
  }
  long pos = 0;
  rp[0] = 0;
  for (int r = 0; r < n; r++) {
    pos += len[r];
    if (pos > 2147483647L) return -1;
    rp[r + 1] = (int)pos;
  }
  return pos;
}

// Columns by Floyd's sampling of rp[r+1]-rp[r] distinct values in
// [0, ncols), sorted ascending; values U[-1,1].  The row's stream continues
// after the length draw made by gen_zipf_rowptr.
void gen_zipf_fill(int n, int ncols, uint64_t seed, const int *rp, int *ci,
                   double *v) {
  #pragma omp parallel
  {
    std::vector<int> pick;
    std::vector<uint8_t> taken((size_t)ncols, 0);  // cleared after each row
    #pragma omp for schedule(dynamic, 1024)
    for (int r = 0; r < n; r++) {
      SplitMix64 g(stream_key(seed, (uint64_t)r));
      (void)g.uniform();  // the length draw
      int L = rp[r + 1] - rp[r];
      pick.clear();
      // Floyd: for j = N-L .. N-1 pick t in [0, j]; take t unless taken,
      // else take j.
      for (int jj = ncols - L; jj < ncols; jj++) {
        int t = (int)(g.next() % (uint64_t)(jj + 1));
        int c = taken[t] ? jj : t;
        taken[c] = 1;
        pick.push_back(c);
      }
      for (int c : pick) taken[c] = 0;
      std::sort(pick.begin(), pick.end());
      long q = rp[r];
      for (int c : pick) {
        ci[q] = c;
        v[q] = 2.0 * g.uniform() - 1.0;
        q++;
      }
    }
  }
}

// Uniform U[lo,hi] vector from a splitmix64 stream per 4096-element block
// (thread-count independent); used for large vectors where the sequential
// mt19937 recipe would dominate setup time.
void gen_uniform_fast_d(long n, double lo, double hi, uint64_t seed,
                        double *out) {
  long nb = (n + 4095) / 4096;
  #pragma omp parallel for schedule(static)
  for (long b = 0; b < nb; b++) {
    SplitMix64 g(stream_key(seed, (uint64_t)b));
    long e = std::min(n, (b + 1) * 4096);
    for (long i = b * 4096; i < e; i++) out[i] = lo + (hi - lo) * g.uniform();
  }
}

// ----------------------------------------------- 3D convection-diffusion
// Interior grid m^3, h = 1/(m+1), diffusion D, velocity s*(1,0.5,0.25) with
// s = 2*D*Pe/h so that max|v_i|*h/(2D) = Pe.  First-order upwind: for each
// axis with v_a > 0 the -1 neighbour carries -(D/h^2 + v_a/h) and the +1
// neighbour -D/h^2; the diagonal is 6D/h^2 + sum_a |v_a|/h.
long gen_convdiff3d_nnz(int m) { return gen_lap3d7p_nnz(m); }
void gen_convdiff3d_fill(int m, double D, double Pe, int *rp, int *ci,
                         double *v) {
  gen_lap3d7p_fill(m, rp, ci, v);  // same structure
  const double h = 1.0 / (m + 1);
  const double s = 2.0 * D * Pe / h;
  const double vel[3] = {s * 1.0, s * 0.5, s * 0.25};  // x (i), y (j), z (k)
  const double dif = D / (h * h);
  const double diag = 6.0 * dif + (std::fabs(vel[0]) + std::fabs(vel[1]) +
                                   std::fabs(vel[2])) / h;
  const long n = (long)m * m * m;
  const long mm = (long)m * m;
  #pragma omp parallel for schedule(static)
  for (long r = 0; r < n; r++) {
    for (long q = rp[r]; q < rp[r + 1]; q++) {
      long c = ci[q];
      long d = c - r;
      int axis = -1;
      int sign = 0;
      if (d == 0) { v[q] = diag; continue; }
      if (d == -1 || d == 1) axis = 0;
      else if (d == -m || d == m) axis = 1;
      else if (d == -mm || d == mm) axis = 2;
      sign = d < 0 ? -1 : 1;
      double va = vel[axis];
      // upwind side: the neighbour the flow comes from
      bool upwind = (va > 0 && sign < 0) || (va < 0 && sign > 0);
      v[q] = upwind ? -(dif + std::fabs(va) / h) : -dif;
    }
  }
}

// ------------------------------------ variable-coefficient diffusion (2D)
long gen_vardiff2d_nnz(int nx, int ny) { return gen_lap2d5p_nnz(nx, ny); }
// Grid nx (fast) by ny; k = exp(N(0,1)) per cell from stream (seed, sys).
void gen_vardiff2d_fill(int nx, int ny, uint64_t seed, uint64_t sys, int *rp,
                        int *ci, double *v) {
  const int n = nx * ny;
  std::vector<double> kc(n);
  SplitMix64 g(stream_key(seed, sys));
  for (int c = 0; c < n; c++) kc[c] = std::exp(g.normal());
  auto face = [&](int a, int b) { return 2.0 * kc[a] * kc[b] / (kc[a] + kc[b]); };
  int q = 0;
  rp[0] = 0;
  for (int c = 0; c < n; c++) {
    int j = c / nx, i = c - j * nx;
    double diag = 0.0;
    int qd;
    if (j > 0) { double f = face(c, c - nx); ci[q] = c - nx; v[q++] = -f; diag += f; }
    else diag += kc[c];
    if (i > 0) { double f = face(c, c - 1); ci[q] = c - 1; v[q++] = -f; diag += f; }
    else diag += kc[c];
    qd = q;
    ci[q] = c; v[q++] = 0.0;
    if (i < nx - 1) { double f = face(c, c + 1); ci[q] = c + 1; v[q++] = -f; diag += f; }
    else diag += kc[c];
    if (j < ny - 1) { double f = face(c, c + nx); ci[q] = c + nx; v[q++] = -f; diag += f; }
    else diag += kc[c];
    v[qd] = diag;
    rp[c + 1] = q;
  }
}

// ------------------------------------ variable-coefficient diffusion (3D)
long gen_vardiff3d_nnz(int nx, int ny, int nz) {
  long n = (long)nx * ny * nz;
  return 7 * n - 2L * ny * nz - 2L * nx * nz - 2L * nx * ny;
}
void gen_vardiff3d_fill(int nx, int ny, int nz, uint64_t seed, uint64_t sys,
                        int *rp, int *ci, double *v) {
  const long n = (long)nx * ny * nz;
  const long pl = (long)nx * ny;
  std::vector<double> kc(n);
  SplitMix64 g(stream_key(seed, sys));
  for (long c = 0; c < n; c++) kc[c] = std::exp(g.normal());
  auto face = [&](long a, long b) { return 2.0 * kc[a] * kc[b] / (kc[a] + kc[b]); };
  long q = 0;
  rp[0] = 0;
  for (long c = 0; c < n; c++) {
    long k = c / pl, j = (c / nx) % ny, i = c % nx;
    double diag = 0.0;
    const long nb[6] = {c - pl, c - nx, c - 1, c + 1, c + nx, c + pl};
    const bool ok[6] = {k > 0, j > 0, i > 0, i < nx - 1, j < ny - 1, k < nz - 1};
    long qd = -1;
    for (int t = 0; t < 6; t++) {
      if (t == 3) { qd = q; ci[q] = (int)c; v[q++] = 0.0; }
      if (ok[t]) {
        double f = face(c, nb[t]);
        ci[q] = (int)nb[t];
        v[q++] = -f;
        diag += f;
      } else {
        diag += kc[c];
      }
    }
    v[qd] = diag;
    rp[c + 1] = (int)q;
  }
}

// ------------------------------------------------- batch / stream sizes
// n_i = round(exp(U[ln lo, ln hi])) from mt19937_64(seed).
void gen_loguniform_sizes(int count, double lo, double hi, uint64_t seed,
                          long *out) {
  std::mt19937_64 mt(seed);
  std::uniform_real_distribution<double> u(std::log(lo), std::log(hi));
  for (int i = 0; i < count; i++) out[i] = std::lround(std::exp(u(mt)));
}

}  // extern "C"
