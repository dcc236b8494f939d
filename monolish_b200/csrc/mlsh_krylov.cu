// Plain CG and BiCGSTAB on one GPU with device-resident scalars.
//
// Reference recurrences kept term for term (no pipelined / s-step
// variants, so iteration counts match the reference's):
//   CG        src/equation/cg.cpp:13-86
//   BiCGSTAB  src/equation/bicgstab.cpp:13-135
//   Jacobi    src/equation/jacobi.cpp:12-61 (M = 1/diag(A), z = M.*r)
//   stopping  ||r||_2 < tol && miniter <= iter, then NaN check
//             (cg.cpp:61-78, equation.cpp:8-11)
//
// Where the reference makes 4-5 host round trips per iteration (every dot
// returns to the host), here every scalar stays on the device: the last CTA
// of each reduction kernel writes it into the handle's SolverState and the
// next kernel reads it.  Per CG iteration there are three kernels:
//   K1  q = A p              fused with (p, q)
//   K2  x += a p, r -= a q   fused with (z, r), (r, r)   [z = M.*r on the fly]
//   K3  p = z + b p          + stopping test in the last CTA
// (BiCGSTAB: five).  The loop body is captured once into a CUDA graph whose
// conditional WHILE node repeats it until the last CTA of K3 clears the
// condition, so a whole solve is one graph launch and one final read.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "mlsh_cluster.cuh"
#include "mlsh_core.cuh"
#include "mlsh_precond.cuh"

namespace mlsh {

template <typename T>
__device__ __forceinline__ double resid_of(double rr) {
  if constexpr (sizeof(T) == 8) {
    return sqrt(rr);
  } else {
    return (double)sqrtf((float)rr);
  }
}

struct CondRef {
  cudaGraphConditionalHandle handle;
  int enabled;
  __device__ void set(int v) const {
    if (enabled) cudaGraphSetConditional(handle, (unsigned)v);
  }
};

// Final bookkeeping of one iteration (CG K3 / BiCGSTAB B5 last CTA).
template <typename T>
__device__ void finish_iteration(SolverState *st, const CondRef &cond) {
  const long long it = st->iter + 1;
  st->iter = it;
  const double res = resid_of<T>(st->rr);
  st->resid = res;
  if (st->hist != nullptr && it <= st->hist_cap) st->hist[it - 1] = res;
  if (res < st->tol && st->miniter <= it) {
    st->status = MLSH_SUCCESS;
    st->done = 1;
  } else if (isnan(res)) {
    st->status = MLSH_SOLVER_RESIDUAL_NAN;
    st->done = 1;
  } else if (it >= st->maxiter) {
    st->status = MLSH_SOLVER_MAXITER;
    st->done = 1;
  }
}

// ------------------------------------------------------------------- CG --
template <typename T, bool JAC>
struct CgInitBody : NoPrep {  // z = M r, p = z; sums (z,r), (r,r)
  const T *r;
  T *p;
  const T *d;
  SolverState *st;
  CondRef cond;
  __device__ void operator()(int64_t i, double *acc) const {
    const T ri = r[i];
    const T zi = JAC ? d[i] * ri : ri;
    p[i] = zi;
    acc[0] += (double)zi * (double)ri;
    acc[1] += (double)ri * (double)ri;
  }
  __device__ void finish(const double *s) {
    st->rz = s[0];
    st->rr = s[1];
    st->resid = resid_of<T>(s[1]);
    if (st->maxiter <= 0) {
      st->status = MLSH_SOLVER_MAXITER;
      st->done = 1;
    }
    cond.set(st->done ? 0 : 1);
  }
};

template <typename T, bool JAC>
struct CgXRBody : NoPrep {  // x += a p; r -= a q; sums (z,r), (r,r)
  T *x;
  T *r;
  const T *p;
  const T *q;
  const T *d;
  SolverState *st;
  T alpha;
  using elem = T;
  bool aligned() const { return al16(x) && al16(r) && al16(p) && al16(q) && (!JAC || al16(d)); }
  __device__ void prepare() { alpha = (T)(st->rz / st->pq); }
  template <int W>
  __device__ void step(int64_t i, double *acc) const {
    const Pack<T, W> pp = ldp<W>(p, i), qq = ldp<W>(q, i);
    Pack<T, W> xx = ldp<W>(x, i), rr = ldp<W>(r, i), dd;
    if (JAC) dd = ldp<W>(d, i);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      xx.v[k] = alpha * pp.v[k] + xx.v[k];
      const T ri = -alpha * qq.v[k] + rr.v[k];
      rr.v[k] = ri;
      const T zi = JAC ? dd.v[k] * ri : ri;
      acc[0] += (double)zi * (double)ri;
      acc[1] += (double)ri * (double)ri;
    }
    stp<W>(x, i, xx);
    stp<W>(r, i, rr);
  }
  __device__ void finish(const double *s) {
    st->rz_new = s[0];
    st->rr = s[1];
  }
};

template <typename T, bool JAC>
struct CgPBody : NoPrep {  // p = z + b p; stopping test
  T *p;
  const T *r;
  const T *d;
  SolverState *st;
  CondRef cond;
  T beta;
  using elem = T;
  bool aligned() const { return al16(p) && al16(r) && (!JAC || al16(d)); }
  __device__ void prepare() { beta = (T)(st->rz_new / st->rz); }
  template <int W>
  __device__ void step(int64_t i, double *) const {
    const Pack<T, W> rr = ldp<W>(r, i);
    Pack<T, W> pp = ldp<W>(p, i), dd;
    if (JAC) dd = ldp<W>(d, i);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const T zi = JAC ? dd.v[k] * rr.v[k] : rr.v[k];
      pp.v[k] = zi + beta * pp.v[k];
    }
    stp<W>(p, i, pp);
  }
  __device__ void finish(const double *) {
    st->rz = st->rz_new;
    finish_iteration<T>(st, cond);
    cond.set(st->done ? 0 : 1);
  }
};

// --------------------------------- CG with a sweep preconditioner -------
// (SOR, IC, ILU: z = M^{-1} r comes from the triangular sweeps, so z is a
// vector of its own and (z, r) a reduction of its own.)
template <typename T>
struct CgInitZBody : NoPrep {  // p = z; sums (z,r), (r,r)
  const T *r;
  const T *z;
  T *p;
  SolverState *st;
  CondRef cond;
  __device__ void operator()(int64_t i, double *acc) const {
    const T ri = r[i], zi = z[i];
    p[i] = zi;
    acc[0] += (double)zi * (double)ri;
    acc[1] += (double)ri * (double)ri;
  }
  __device__ void finish(const double *s) {
    st->rz = s[0];
    st->rr = s[1];
    st->resid = resid_of<T>(s[1]);
    if (st->maxiter <= 0) {
      st->status = MLSH_SOLVER_MAXITER;
      st->done = 1;
    }
    cond.set(st->done ? 0 : 1);
  }
};

template <typename T>
struct ZRBody : NoPrep {  // (z, r) of the preconditioned residual
  const T *z;
  const T *r;
  SolverState *st;
  using elem = T;
  bool aligned() const { return al16(z) && al16(r); }
  template <int W>
  __device__ void step(int64_t i, double *acc) const {
    const Pack<T, W> zz = ldp<W>(z, i), rr = ldp<W>(r, i);
#pragma unroll
    for (int k = 0; k < W; ++k) acc[0] += (double)zz.v[k] * (double)rr.v[k];
  }
  __device__ void finish(const double *s) { st->rz_new = s[0]; }
};

// ------------------------------------------------------------------ SOR --
// equation::SOR::solve (src/equation/sor.cpp:92-162): per iteration
// r = b - A x, t = (D/omega + L)^{-1} r, x += t, then the test on
// ||r|| / ||b||.
template <typename T>
struct SorInitBody : NoPrep {  // 1 / ||b||  (sor.cpp:118-119)
  const T *b;
  SolverState *st;
  CondRef cond;
  __device__ void operator()(int64_t i, double *acc) const {
    const double v = (double)b[i];
    acc[0] += v * v;
  }
  __device__ void finish(const double *s) {
    const T nb = (T)resid_of<T>(s[0]);
    st->scale = (double)(T)(1.0 / (double)nb);
    st->resid = 0.0;
    if (st->maxiter <= 0) {
      st->status = MLSH_SOLVER_MAXITER;
      st->done = 1;
    }
    cond.set(st->done ? 0 : 1);
  }
};

template <typename T>
struct SorXBody : NoPrep {  // x += t; stopping test (sor.cpp:137-157)
  T *x;
  const T *t;
  SolverState *st;
  CondRef cond;
  using elem = T;
  bool aligned() const { return al16(x) && al16(t); }
  template <int W>
  __device__ void step(int64_t i, double *) const {
    const Pack<T, W> tt = ldp<W>(t, i);
    Pack<T, W> xx = ldp<W>(x, i);
#pragma unroll
    for (int k = 0; k < W; ++k) xx.v[k] = tt.v[k] + xx.v[k];
    stp<W>(x, i, xx);
  }
  __device__ void finish(const double *) {
    const long long it = st->iter + 1;
    st->iter = it;
    const T nrm = (T)resid_of<T>(st->rr);
    const T rel = nrm * (T)st->scale;
    st->resid = (double)nrm;  // final_resid = get_residual(r), absolute
    if (st->hist != nullptr && it <= st->hist_cap) st->hist[it - 1] = (double)rel;
    if ((double)rel < st->tol && st->miniter <= it) {
      st->status = MLSH_SUCCESS;
      st->done = 1;
    } else if (isnan(rel)) {
      st->status = MLSH_SOLVER_RESIDUAL_NAN;
      st->done = 1;
    } else if (it >= st->maxiter) {
      st->status = MLSH_SOLVER_MAXITER;
      st->done = 1;
    }
    cond.set(st->done ? 0 : 1);
  }
};

// ------------------------------------------------------------- BiCGSTAB --
template <typename T>
__device__ void bicg_rho_check(SolverState *st) {
  // start of the next iteration: rho = (r, r0) == 0 -> breakdown
  // (bicgstab.cpp:56-63); final_iter is that iteration's index + 1.
  if (!st->done && st->rho == 0.0) {
    st->status = MLSH_SOLVER_BREAKDOWN;
    st->done = 1;
    st->iter = st->iter + 1;
  }
}

template <typename T>
struct BiInitBody : NoPrep {  // r0 = r; sums (r, r0), (r, r)
  const T *r;
  T *r0;
  SolverState *st;
  CondRef cond;
  __device__ void operator()(int64_t i, double *acc) const {
    const T ri = r[i];
    r0[i] = ri;
    acc[0] += (double)ri * (double)ri;
    acc[1] += (double)ri * (double)ri;
  }
  __device__ void finish(const double *s) {
    st->rho = s[0];
    st->rr = s[1];
    st->rho_old = 1.0;
    st->alpha = 1.0;
    st->omega = 1.0;
    st->resid = resid_of<T>(s[1]);
    if (st->maxiter <= 0) {
      st->status = MLSH_SOLVER_MAXITER;
      st->done = 1;
    } else {
      bicg_rho_check<T>(st);
    }
    cond.set(st->done ? 0 : 1);
  }
};

template <typename T, bool JAC>
struct BiPBody : NoPrep {  // p = r + beta (p - omega v); phat = M p
  const T *r;
  T *p;
  const T *v;
  T *phat;
  const T *d;
  SolverState *st;
  T beta, omega;
  int first;
  using elem = T;
  bool aligned() const { return al16(r) && al16(p) && al16(v) && al16(phat) && (!JAC || al16(d)); }
  __device__ void prepare() {
    first = st->iter == 0;
    omega = (T)st->omega;
    beta = (T)((st->rho / st->rho_old) * (st->alpha / st->omega));
  }
  template <int W>
  __device__ void step(int64_t i, double *) const {
    const Pack<T, W> rr = ldp<W>(r, i);
    Pack<T, W> pp;
    if (first) {
      pp = rr;
    } else {
      const Pack<T, W> vv = ldp<W>(v, i);
      pp = ldp<W>(p, i);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const T t = -omega * vv.v[k] + pp.v[k];
        pp.v[k] = rr.v[k] + beta * t;
      }
    }
    stp<W>(p, i, pp);
    if (JAC) {
      Pack<T, W> dd = ldp<W>(d, i);
#pragma unroll
      for (int k = 0; k < W; ++k) dd.v[k] = dd.v[k] * pp.v[k];
      stp<W>(phat, i, dd);
    }
  }
};

template <typename T, bool JAC>
struct BiSBody : NoPrep {  // alpha = rho/(v,r0); s = r - alpha v; shat = M s
  const T *r;
  const T *v;
  T *s;
  T *shat;
  const T *d;
  SolverState *st;
  T alpha;
  double alpha_d;
  using elem = T;
  bool aligned() const { return al16(r) && al16(v) && al16(s) && al16(shat) && (!JAC || al16(d)); }
  __device__ void prepare() {
    alpha_d = st->rho / st->vr0;
    alpha = (T)alpha_d;
  }
  template <int W>
  __device__ void step(int64_t i, double *) const {
    const Pack<T, W> vv = ldp<W>(v, i), rr = ldp<W>(r, i);
    Pack<T, W> ss;
#pragma unroll
    for (int k = 0; k < W; ++k) ss.v[k] = -alpha * vv.v[k] + rr.v[k];
    stp<W>(s, i, ss);
    if (JAC) {
      Pack<T, W> dd = ldp<W>(d, i);
#pragma unroll
      for (int k = 0; k < W; ++k) dd.v[k] = dd.v[k] * ss.v[k];
      stp<W>(shat, i, dd);
    }
  }
  __device__ void finish(const double *) { st->alpha = (double)alpha; }
};

template <typename T>
struct BiXRBody : NoPrep {  // omega = (t,s)/(t,t); x += a phat + w shat; r = s - w t
  T *x;
  T *r;
  const T *r0;
  const T *phat;
  const T *shat;
  const T *s;
  const T *t;
  SolverState *st;
  CondRef cond;
  T alpha, omega;
  int brk;
  using elem = T;
  bool aligned() const {
    return al16(x) && al16(r) && al16(r0) && al16(phat) && al16(shat) && al16(s) && al16(t);
  }
  __device__ void prepare() {
    omega = (T)(st->ts / st->tt);
    alpha = (T)st->alpha;
    brk = (omega == T(0));
  }
  template <int W>
  __device__ void step(int64_t i, double *acc) const {
    if (brk) return;
    const Pack<T, W> ph = ldp<W>(phat, i), sh = ldp<W>(shat, i), tt = ldp<W>(t, i),
                     ss = ldp<W>(s, i), rz = ldp<W>(r0, i);
    Pack<T, W> xx = ldp<W>(x, i), rr;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      T xi = alpha * ph.v[k] + xx.v[k];
      xx.v[k] = omega * sh.v[k] + xi;
      const T ri = -omega * tt.v[k] + ss.v[k];
      rr.v[k] = ri;
      acc[0] += (double)ri * (double)rz.v[k];
      acc[1] += (double)ri * (double)ri;
    }
    stp<W>(x, i, xx);
    stp<W>(r, i, rr);
  }
  __device__ void finish(const double *sums) {
    if (brk) {
      // bicgstab.cpp:93-98: breakdown before x and r are updated
      st->status = MLSH_SOLVER_BREAKDOWN;
      st->done = 1;
      st->iter = st->iter + 1;
      st->resid = resid_of<T>(st->rr);
    } else {
      st->omega = (double)omega;
      st->rho_old = st->rho;
      st->rho = sums[0];
      st->rr = sums[1];
      finish_iteration<T>(st, cond);
      bicg_rho_check<T>(st);
    }
    cond.set(st->done ? 0 : 1);
  }
};

// ------------------------------------------ mixed precision, BiCGSTAB --
// FP32 BiCGSTAB iterations on A32 with reliable updates (Sleijpen & van der
// Vorst, "Reliable updated residuals in hybrid Bi-CG methods", Computing
// 56 (1996); the mixed-precision form of Clark et al., Comput. Phys. Commun.
// 181 (2010)): the FP32 iterate x32 holds the correction since the last
// update; whenever the iterated residual has dropped by `delta` since the
// last true residual (or the iteration ends), x += scale * x32 in FP64, the
// true residual b - A x is formed with the FP64 matrix, and the FP32
// iteration continues from it without restarting its Krylov space.  The
// stopping test is on the true FP64 residual.

// Initial pass: r32 = r64 / s, r0 = r32, x32 = 0 with s = ||r64||.
struct MixInitBody {
  const double *r64;
  float *r32;
  float *r0;
  float *x32;
  SolverState *st;
  CondRef cond;
  double inv;
  __device__ void prepare() { inv = st->rr64 > 0.0 ? 1.0 / sqrt(st->rr64) : 1.0; }
  __device__ void operator()(int64_t i, double *acc) const {
    const float r = (float)(r64[i] * inv);
    r32[i] = r;
    r0[i] = r;
    x32[i] = 0.0f;
    acc[0] += (double)r * (double)r;
    acc[1] += (double)r * (double)r;
  }
  __device__ void finish(const double *s) {
    const double tr = sqrt(st->rr64);
    st->scale = tr > 0.0 ? tr : 1.0;
    st->rel_true = tr;
    st->resid = tr;
    st->outer = 0;
    if (st->hist != nullptr && st->hist_cap > 0) st->hist[0] = tr;
    st->rho = s[0];
    st->rr = s[1];
    st->rho_old = st->alpha = st->omega = 1.0;
    st->first = 1;
    st->upd = 0;
    st->noupd = 1;
    st->pending = kRunning;
    if (st->maxiter <= 0) {
      st->status = MLSH_SOLVER_MAXITER;
      st->done = 1;
    } else if (tr < st->tol && st->miniter <= 0) {
      st->status = MLSH_SUCCESS;
      st->done = 1;
    } else if (isnan(tr)) {
      st->status = MLSH_SOLVER_RESIDUAL_NAN;
      st->done = 1;
    }
    cond.set(st->done ? 0 : 1);
  }
};

// Update, part 1: x += s * D^-1 x32 (FP64; D^-1 = 1 without Jacobi), x32 = 0.
struct MixXUpdBody : NoPrep {
  double *x64;
  float *x32;
  const double *dinv;  // Jacobi: the FP32 iteration runs on A D^-1 (right scaling)
  SolverState *st;
  double s;
  __device__ void prepare() { s = st->scale; }
  __device__ void operator()(int64_t i, double *) const {
    const double c = dinv != nullptr ? s * dinv[i] : s;
    x64[i] = c * (double)x32[i] + x64[i];
    x32[i] = 0.0f;
  }
};

// Update, part 3 (after r64 = b - A x in FP64): r32 = r64 / s; a fresh
// Krylov space also restarts the shadow residual r0 = r32.
struct MixRUpdBody {
  const double *r64;
  float *r32;
  float *r0;
  SolverState *st;
  CondRef cond;
  double inv;
  int fresh;
  __device__ void prepare() {
    inv = 1.0 / st->scale;
    fresh = st->first;
  }
  __device__ void operator()(int64_t i, double *acc) const {
    const float r = (float)(r64[i] * inv);
    r32[i] = r;
    float z;
    if (fresh) {
      r0[i] = r;
      z = r;
    } else {
      z = r0[i];
    }
    acc[0] += (double)r * (double)z;
    acc[1] += (double)r * (double)r;
  }
  __device__ void finish(const double *s) {
    const double tr = sqrt(st->rr64);
    const long long o = st->outer + 1;
    st->outer = o;
    if (st->hist != nullptr && o < st->hist_cap) st->hist[o] = tr;
    st->resid = tr;
    st->rel_true = tr;
    st->upd = 0;
    st->noupd = 1;
    if (tr < st->tol && st->miniter <= st->iter) {
      st->status = MLSH_SUCCESS;
      st->done = 1;
    } else if (isnan(tr)) {
      st->status = MLSH_SOLVER_RESIDUAL_NAN;
      st->done = 1;
    } else if (st->pending != kRunning) {
      st->status = st->pending;
      st->done = 1;
    } else {
      st->rho = s[0];
      st->rr = s[1];
      if (s[0] == 0.0) {  // r orthogonal to r0: nothing to continue from
        st->status = MLSH_SOLVER_BREAKDOWN;
        st->done = 1;
      }
    }
    cond.set(st->done ? 0 : 1);
  }
};

template <bool JAC>
struct MixPBody {  // p = r + beta (p - omega v) (or p = r on a fresh start); phat = M p
  const float *r;
  float *p;
  const float *v;
  float *phat;
  const float *d;
  SolverState *st;
  float beta, omega;
  int first;
  using elem = float;
  bool aligned() const { return al16(r) && al16(p) && al16(v) && al16(phat) && (!JAC || al16(d)); }
  __device__ void prepare() {
    first = st->first;
    omega = (float)st->omega;
    beta = (float)((st->rho / st->rho_old) * (st->alpha / st->omega));
  }
  template <int W>
  __device__ void step(int64_t i, double *) const {
    const Pack<float, W> rr = ldp<W>(r, i);
    Pack<float, W> pp;
    if (first) {
      pp = rr;
    } else {
      const Pack<float, W> vv = ldp<W>(v, i);
      pp = ldp<W>(p, i);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const float t = -omega * vv.v[k] + pp.v[k];
        pp.v[k] = rr.v[k] + beta * t;
      }
    }
    stp<W>(p, i, pp);
    if (JAC) {
      Pack<float, W> dd = ldp<W>(d, i);
#pragma unroll
      for (int k = 0; k < W; ++k) dd.v[k] = dd.v[k] * pp.v[k];
      stp<W>(phat, i, dd);
    }
  }
  __device__ void finish(const double *) { st->first = 0; }
};

struct MixXRBody : NoPrep {  // x32 += a phat + w shat; r = s - w t; decide on an update
  float *x;
  float *r;
  const float *r0;
  const float *phat;
  const float *shat;
  const float *s;
  const float *t;
  SolverState *st;
  CondRef upd_cond;
  float alpha, omega;
  int brk;
  using elem = float;
  bool aligned() const {
    return al16(x) && al16(r) && al16(r0) && al16(phat) && al16(shat) && al16(s) && al16(t);
  }
  __device__ void prepare() {
    omega = (float)(st->ts / st->tt);
    alpha = (float)st->alpha;
    brk = (omega == 0.0f);
  }
  template <int W>
  __device__ void step(int64_t i, double *acc) const {
    if (brk) return;
    const Pack<float, W> ph = ldp<W>(phat, i), sh = ldp<W>(shat, i), tt = ldp<W>(t, i),
                     ss = ldp<W>(s, i), rz = ldp<W>(r0, i);
    Pack<float, W> xx = ldp<W>(x, i), rr;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      float xi = alpha * ph.v[k] + xx.v[k];
      xx.v[k] = omega * sh.v[k] + xi;
      const float ri = -omega * tt.v[k] + ss.v[k];
      rr.v[k] = ri;
      acc[0] += (double)ri * (double)rz.v[k];
      acc[1] += (double)ri * (double)ri;
    }
    stp<W>(x, i, xx);
    stp<W>(r, i, rr);
  }
  __device__ void finish(const double *sums) {
    const long long it = st->iter + 1;
    st->iter = it;
    int upd = 0;
    if (brk) {
      // omega = 0: apply the correction so far and restart the Krylov space
      st->first = 1;
      upd = 1;
    } else {
      st->omega = (double)omega;
      st->rho_old = st->rho;
      st->rho = sums[0];
      st->rr = sums[1];
      const double res = (double)sqrtf((float)sums[1]) * st->scale;
      if (isnan(res)) {
        st->pending = MLSH_SOLVER_RESIDUAL_NAN;
        upd = 1;
      } else if (res < st->delta * st->rel_true || res < st->tol) {
        upd = 1;
      } else if (sums[0] == 0.0) {
        st->first = 1;
        upd = 1;
      }
    }
    if (!upd && it >= st->maxiter) upd = 1;
    if (it >= st->maxiter && st->pending == kRunning) st->pending = MLSH_SOLVER_MAXITER;
    st->upd = upd;
    st->noupd = 1 - upd;
    upd_cond.set(upd);
  }
};

// --------------------------------------------------------------- driver --
namespace {

// CTAs of a packed launch: at most one wave of the kernel's resident CTAs
// (a second partial wave would leave most SMs idle at its end).
template <auto kernel>
int pack_grid(int64_t n, int w, int num_sms) {
  static int per_sm = 0;  // one value per kernel
  if (per_sm == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kVecThreads, 0) !=
            cudaSuccess ||
        b < 1) {
      cudaGetLastError();
      b = 1;
    }
    per_sm = std::min(b, kMaxVecBlocksPerSm);
  }
  int64_t g = (n + (int64_t)kVecThreads * w * 4 - 1) / ((int64_t)kVecThreads * w * 4);
  g = std::min<int64_t>(g, (int64_t)per_sm * num_sms);
  return (int)std::max<int64_t>(g, 1);
}

template <int NR, bool FIN, typename Body>
cudaError_t run_body(const Handle &h, int64_t n, const Body &b, const int *done,
                     cudaStream_t s) {
  RedArgs ra{h.partials, h.counters, done};
  const int g = vec_grid(n, h.num_sms);
  if constexpr (has_step<Body>::value) {
    constexpr int W = 16 / (int)sizeof(typename Body::elem);
    if (b.aligned()) {
      constexpr auto k = vec_pack_kernel<NR, FIN, W, Body>;
      return launch_dependent(k, pack_grid<k>(n, W, h.num_sms), kVecThreads, 0, s, n, b, ra);
    }
    constexpr auto k = vec_pack_kernel<NR, FIN, 1, Body>;
    return launch_dependent(k, pack_grid<k>(n, 1, h.num_sms), kVecThreads, 0, s, n, b, ra);
  } else {
    return launch_dependent(vec_kernel<NR, FIN, Body>, g, kVecThreads, 0, s, n, b, ra);
  }
}

enum Kind { kCG = 0, kBiCGSTAB = 1, kMixedBiCGSTAB = 3, kSOR = 4 };

struct SolveCtx {
  Kind kind;
  int dtype;
  int jac;
  const CsrPlan *plan;
  const Handle *h;
  const void *b;
  void *x;
  const void *d;  // inverse diagonal (Jacobi) or null
  void *ws;       // work vectors, `stride` elements apart
  int64_t n;
  int64_t stride;
  // mixed kinds: `plan` is the FP32 copy, `b`/`x` are FP64, and
  const CsrPlan *plan64 = nullptr;  // the FP64 matrix
  double *r64 = nullptr;            // FP64 residual vector
  CondRef upd_cond = {0, 0};        // graph: the IF node that runs the update
  // sweep preconditioner (SOR / IC / ILU), or for kSOR the solver's sweep
  const Precond *pc = nullptr;
};

template <typename T>
T *wsv(const SolveCtx &c, int k) {
  return static_cast<T *>(c.ws) + (size_t)k * (size_t)c.stride;
}

// ---- CG
template <typename T, bool JAC>
cudaError_t cg_init(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *p = wsv<T>(c, 1);
  cudaError_t e = launch_spmv_t<T, kDotNone, kDotNone>(
      *c.plan, *c.h, -1.0, static_cast<const T *>(c.x), 1.0,
      static_cast<const T *>(c.b), r, nullptr, nullptr, nullptr, nullptr, s);
  if (e != cudaSuccess) return e;
  CgInitBody<T, JAC> ib;
  ib.r = r; ib.p = p; ib.d = static_cast<const T *>(c.d); ib.st = c.h->state; ib.cond = cond;
  return run_body<2, true>(*c.h, c.n, ib, nullptr, s);
}

template <typename T, bool JAC>
cudaError_t cg_iter(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *p = wsv<T>(c, 1), *q = wsv<T>(c, 2);
  SolverState *st = c.h->state;
  const int *done = &st->done;
  cudaError_t e = launch_spmv_t<T, kDotW, kDotNone>(*c.plan, *c.h, 1.0, p, 0.0, nullptr, q,
                                                    p, nullptr, &st->pq, done, s);
  if (e != cudaSuccess) return e;
  CgXRBody<T, JAC> xb;
  xb.x = static_cast<T *>(c.x); xb.r = r; xb.p = p; xb.q = q;
  xb.d = static_cast<const T *>(c.d); xb.st = st;
  e = run_body<2, true>(*c.h, c.n, xb, done, s);
  if (e != cudaSuccess) return e;
  CgPBody<T, JAC> pb;
  pb.p = p; pb.r = r; pb.d = static_cast<const T *>(c.d); pb.st = st; pb.cond = cond;
  return run_body<0, true>(*c.h, c.n, pb, done, s);
}

// ---- BiCGSTAB: ws = r, r0, p, v, s, t, phat, shat
template <typename T, bool JAC>
cudaError_t bi_init(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *r0 = wsv<T>(c, 1);
  cudaError_t e = launch_spmv_t<T, kDotNone, kDotNone>(
      *c.plan, *c.h, -1.0, static_cast<const T *>(c.x), 1.0,
      static_cast<const T *>(c.b), r, nullptr, nullptr, nullptr, nullptr, s);
  if (e != cudaSuccess) return e;
  BiInitBody<T> ib;
  ib.r = r; ib.r0 = r0; ib.st = c.h->state; ib.cond = cond;
  return run_body<2, true>(*c.h, c.n, ib, nullptr, s);
}

template <typename T, bool JAC>
cudaError_t bi_iter(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *r0 = wsv<T>(c, 1), *p = wsv<T>(c, 2), *v = wsv<T>(c, 3);
  T *sv = wsv<T>(c, 4), *t = wsv<T>(c, 5);
  T *phat = JAC ? wsv<T>(c, 6) : p;
  T *shat = JAC ? wsv<T>(c, 7) : sv;
  const T *d = static_cast<const T *>(c.d);
  SolverState *st = c.h->state;
  const int *done = &st->done;
  BiPBody<T, JAC> pb;
  pb.r = r; pb.p = p; pb.v = v; pb.phat = phat; pb.d = d; pb.st = st;
  cudaError_t e = run_body<0, false>(*c.h, c.n, pb, done, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<T, kDotW, kDotNone>(*c.plan, *c.h, 1.0, phat, 0.0, nullptr, v, r0,
                                        nullptr, &st->vr0, done, s);
  if (e != cudaSuccess) return e;
  BiSBody<T, JAC> sb;
  sb.r = r; sb.v = v; sb.s = sv; sb.shat = shat; sb.d = d; sb.st = st;
  e = run_body<0, true>(*c.h, c.n, sb, done, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<T, kDotW, kDotSelf>(*c.plan, *c.h, 1.0, shat, 0.0, nullptr, t, sv,
                                        nullptr, &st->ts, done, s);
  if (e != cudaSuccess) return e;
  BiXRBody<T> xb;
  xb.x = static_cast<T *>(c.x); xb.r = r; xb.r0 = r0; xb.phat = phat; xb.shat = shat;
  xb.s = sv; xb.t = t; xb.st = st; xb.cond = cond;
  return run_body<2, true>(*c.h, c.n, xb, done, s);
}

// ---- CG with a sweep preconditioner: ws = r, p, q, z
template <typename T>
cudaError_t cgf_init(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *p = wsv<T>(c, 1), *z = wsv<T>(c, 3);
  cudaError_t e = launch_spmv_t<T, kDotNone, kDotNone>(
      *c.plan, *c.h, -1.0, static_cast<const T *>(c.x), 1.0,
      static_cast<const T *>(c.b), r, nullptr, nullptr, nullptr, nullptr, s);
  if (e != cudaSuccess) return e;
  e = precond_apply_launch(*c.pc, r, z, nullptr, c.h->err_flag, s);
  if (e != cudaSuccess) return e;
  CgInitZBody<T> ib;
  ib.r = r; ib.z = z; ib.p = p; ib.st = c.h->state; ib.cond = cond;
  return run_body<2, true>(*c.h, c.n, ib, nullptr, s);
}

template <typename T>
cudaError_t cgf_iter(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *p = wsv<T>(c, 1), *q = wsv<T>(c, 2), *z = wsv<T>(c, 3);
  SolverState *st = c.h->state;
  const int *done = &st->done;
  cudaError_t e = launch_spmv_t<T, kDotW, kDotNone>(*c.plan, *c.h, 1.0, p, 0.0, nullptr, q,
                                                    p, nullptr, &st->pq, done, s);
  if (e != cudaSuccess) return e;
  CgXRBody<T, false> xb;
  xb.x = static_cast<T *>(c.x); xb.r = r; xb.p = p; xb.q = q; xb.d = nullptr; xb.st = st;
  e = run_body<2, true>(*c.h, c.n, xb, done, s);
  if (e != cudaSuccess) return e;
  e = precond_apply_launch(*c.pc, r, z, done, c.h->err_flag, s);
  if (e != cudaSuccess) return e;
  ZRBody<T> zb;
  zb.z = z; zb.r = r; zb.st = st;
  e = run_body<1, true>(*c.h, c.n, zb, done, s);
  if (e != cudaSuccess) return e;
  CgPBody<T, false> pb;
  pb.p = p; pb.r = z; pb.d = nullptr; pb.st = st; pb.cond = cond;
  return run_body<0, true>(*c.h, c.n, pb, done, s);
}

// ---- BiCGSTAB with a sweep preconditioner: ws = r, r0, p, v, s, t, phat, shat
template <typename T>
cudaError_t bif_iter(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *r0 = wsv<T>(c, 1), *p = wsv<T>(c, 2), *v = wsv<T>(c, 3);
  T *sv = wsv<T>(c, 4), *t = wsv<T>(c, 5), *phat = wsv<T>(c, 6), *shat = wsv<T>(c, 7);
  SolverState *st = c.h->state;
  const int *done = &st->done;
  BiPBody<T, false> pb;
  pb.r = r; pb.p = p; pb.v = v; pb.phat = p; pb.d = nullptr; pb.st = st;
  cudaError_t e = run_body<0, false>(*c.h, c.n, pb, done, s);
  if (e != cudaSuccess) return e;
  e = precond_apply_launch(*c.pc, p, phat, done, c.h->err_flag, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<T, kDotW, kDotNone>(*c.plan, *c.h, 1.0, phat, 0.0, nullptr, v, r0,
                                        nullptr, &st->vr0, done, s);
  if (e != cudaSuccess) return e;
  BiSBody<T, false> sb;
  sb.r = r; sb.v = v; sb.s = sv; sb.shat = sv; sb.d = nullptr; sb.st = st;
  e = run_body<0, true>(*c.h, c.n, sb, done, s);
  if (e != cudaSuccess) return e;
  e = precond_apply_launch(*c.pc, sv, shat, done, c.h->err_flag, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<T, kDotW, kDotSelf>(*c.plan, *c.h, 1.0, shat, 0.0, nullptr, t, sv,
                                        nullptr, &st->ts, done, s);
  if (e != cudaSuccess) return e;
  BiXRBody<T> xb;
  xb.x = static_cast<T *>(c.x); xb.r = r; xb.r0 = r0; xb.phat = phat; xb.shat = shat;
  xb.s = sv; xb.t = t; xb.st = st; xb.cond = cond;
  return run_body<2, true>(*c.h, c.n, xb, done, s);
}

// ---- SOR: ws = r, t
template <typename T>
cudaError_t sor_init(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  SorInitBody<T> ib;
  ib.b = static_cast<const T *>(c.b); ib.st = c.h->state; ib.cond = cond;
  return run_body<1, true>(*c.h, c.n, ib, nullptr, s);
}

template <typename T>
cudaError_t sor_iter(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  T *r = wsv<T>(c, 0), *t = wsv<T>(c, 1);
  SolverState *st = c.h->state;
  const int *done = &st->done;
  cudaError_t e = launch_spmv_t<T, kDotSelf, kDotNone>(
      *c.plan, *c.h, -1.0, static_cast<const T *>(c.x), 1.0, static_cast<const T *>(c.b), r,
      nullptr, nullptr, &st->rr, done, s);
  if (e != cudaSuccess) return e;
  e = sweep_launch(*c.pc, c.pc->fwd, false, r, t, done, c.h->err_flag, s);
  if (e != cudaSuccess) return e;
  SorXBody<T> xb;
  xb.x = static_cast<T *>(c.x); xb.t = t; xb.st = st; xb.cond = cond;
  return run_body<0, true>(*c.h, c.n, xb, done, s);
}

// ---- mixed BiCGSTAB: ws (FP32) = r, r0, p, v, s, t, x32.  With Jacobi the
// FP32 matrix holds A D^-1 (right preconditioning folded into the values),
// so the FP32 iteration itself is unpreconditioned and c.d is the FP64
// inverse diagonal the update applies.
cudaError_t mixbi_init(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  SolverState *st = c.h->state;
  cudaError_t e = launch_spmv_t<double, kDotSelf, kDotNone>(
      *c.plan64, *c.h, -1.0, static_cast<const double *>(c.x), 1.0,
      static_cast<const double *>(c.b), c.r64, nullptr, nullptr, &st->rr64, nullptr, s);
  if (e != cudaSuccess) return e;
  MixInitBody ib;
  ib.r64 = c.r64; ib.r32 = wsv<float>(c, 0); ib.r0 = wsv<float>(c, 1);
  ib.x32 = wsv<float>(c, 6); ib.st = st; ib.cond = cond;
  return run_body<2, true>(*c.h, c.n, ib, nullptr, s);
}

// One FP32 BiCGSTAB iteration; its last kernel decides whether an update
// follows.
cudaError_t mixbi_main(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  (void)cond;
  float *r = wsv<float>(c, 0), *r0 = wsv<float>(c, 1), *p = wsv<float>(c, 2);
  float *v = wsv<float>(c, 3), *sv = wsv<float>(c, 4), *t = wsv<float>(c, 5);
  float *x32 = wsv<float>(c, 6);
  SolverState *st = c.h->state;
  const int *done = &st->done;
  MixPBody<false> pb;
  pb.r = r; pb.p = p; pb.v = v; pb.phat = p; pb.d = nullptr; pb.st = st;
  cudaError_t e = run_body<0, true>(*c.h, c.n, pb, done, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<float, kDotW, kDotNone>(*c.plan, *c.h, 1.0, p, 0.0, nullptr, v, r0,
                                            nullptr, &st->vr0, done, s);
  if (e != cudaSuccess) return e;
  BiSBody<float, false> sb;
  sb.r = r; sb.v = v; sb.s = sv; sb.shat = sv; sb.d = nullptr; sb.st = st;
  e = run_body<0, true>(*c.h, c.n, sb, done, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<float, kDotW, kDotSelf>(*c.plan, *c.h, 1.0, sv, 0.0, nullptr, t, sv,
                                            nullptr, &st->ts, done, s);
  if (e != cudaSuccess) return e;
  MixXRBody xb;
  xb.x = x32; xb.r = r; xb.r0 = r0; xb.phat = p; xb.shat = sv; xb.s = sv; xb.t = t;
  xb.st = st; xb.upd_cond = c.upd_cond;
  return run_body<2, true>(*c.h, c.n, xb, done, s);
}

// The reliable update: x += s D^-1 x32, r64 = b - A x (FP64), r32 = r64 / s.
// In a graph it sits under an IF node; launched one by one, each kernel
// skips itself unless an update is pending.
cudaError_t mixbi_update(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  float *r = wsv<float>(c, 0), *r0 = wsv<float>(c, 1), *x32 = wsv<float>(c, 6);
  SolverState *st = c.h->state;
  const int *skip = c.upd_cond.enabled ? nullptr : &st->noupd;
  MixXUpdBody ub;
  ub.x64 = static_cast<double *>(c.x); ub.x32 = x32;
  ub.dinv = static_cast<const double *>(c.d); ub.st = st;
  cudaError_t e = run_body<0, false>(*c.h, c.n, ub, skip, s);
  if (e != cudaSuccess) return e;
  e = launch_spmv_t<double, kDotSelf, kDotNone>(
      *c.plan64, *c.h, -1.0, static_cast<const double *>(c.x), 1.0,
      static_cast<const double *>(c.b), c.r64, nullptr, nullptr, &st->rr64, skip, s);
  if (e != cudaSuccess) return e;
  MixRUpdBody rb;
  rb.r64 = c.r64; rb.r32 = r; rb.r0 = r0; rb.st = st; rb.cond = cond;
  return run_body<2, true>(*c.h, c.n, rb, skip, s);
}

cudaError_t mixbi_iter(const SolveCtx &c, cudaStream_t s, CondRef cond) {
  cudaError_t e = mixbi_main(c, s, cond);
  if (e != cudaSuccess) return e;
  return mixbi_update(c, s, cond);
}

using StepFn = cudaError_t (*)(const SolveCtx &, cudaStream_t, CondRef);

void pick_steps(const SolveCtx &c, StepFn *init, StepFn *iter) {
  const bool f64 = c.dtype == MLSH_F64;
  if (c.kind == kMixedBiCGSTAB) {
    *init = mixbi_init;
    *iter = mixbi_iter;
    return;
  }
  if (c.pc != nullptr) {
    if (c.kind == kSOR) {
      *init = f64 ? sor_init<double> : sor_init<float>;
      *iter = f64 ? sor_iter<double> : sor_iter<float>;
    } else if (c.kind == kCG) {
      *init = f64 ? cgf_init<double> : cgf_init<float>;
      *iter = f64 ? cgf_iter<double> : cgf_iter<float>;
    } else {
      *init = f64 ? bi_init<double, false> : bi_init<float, false>;
      *iter = f64 ? bif_iter<double> : bif_iter<float>;
    }
    return;
  }
  if (c.kind == kCG) {
    if (f64) {
      *init = c.jac ? cg_init<double, true> : cg_init<double, false>;
      *iter = c.jac ? cg_iter<double, true> : cg_iter<double, false>;
    } else {
      *init = c.jac ? cg_init<float, true> : cg_init<float, false>;
      *iter = c.jac ? cg_iter<float, true> : cg_iter<float, false>;
    }
  } else {
    if (f64) {
      *init = c.jac ? bi_init<double, true> : bi_init<double, false>;
      *iter = c.jac ? bi_iter<double, true> : bi_iter<double, false>;
    } else {
      *init = c.jac ? bi_init<float, true> : bi_init<float, false>;
      *iter = c.jac ? bi_iter<float, true> : bi_iter<float, false>;
    }
  }
}

// ------------------------------------------------------- graph cache ----
struct GraphEntry {
  Kind kind;
  int dtype, jac;
  const CsrPlan *plan;
  const void *b;
  void *x;
  const void *d;
  void *ws;
  int64_t n;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  unsigned long long last_use;
  const Precond *pc;
};

struct GraphCache {
  std::vector<GraphEntry> entries;
  unsigned long long clock = 0;
};

GraphCache &cache_of(Handle &h) {
  if (!h.graph_cache) h.graph_cache = new GraphCache();
  return *static_cast<GraphCache *>(h.graph_cache);
}

void destroy_entry(GraphEntry &e) {
  if (e.exec) cudaGraphExecDestroy(e.exec);
  if (e.graph) cudaGraphDestroy(e.graph);
  e.exec = nullptr;
  e.graph = nullptr;
}

// Builds  [init kernels] -> WHILE(cond) { one iteration }  as one graph.
int build_graph(const SolveCtx &c, Handle &h, GraphEntry &out) {
  StepFn init, iter;
  pick_steps(c, &init, &iter);
  cudaGraph_t g = nullptr;
  MLSH_CUDA_TRY(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle cond;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_last_error("cudaGraphConditionalHandleCreate", e);
    return MLSH_ERR_CUDA;
  }
  CondRef cr{cond, 1};
  // init part, captured into g
  e = cudaStreamBeginCaptureToGraph(h.capture_stream, g, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t e2 = init(c, h.capture_stream, cr);
    cudaGraph_t gg = nullptr;
    e = cudaStreamEndCapture(h.capture_stream, &gg);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_last_error("capture solver init", e);
    return MLSH_ERR_CUDA;
  }
  // leaves of the init part
  size_t nn = 0;
  cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn), leaves;
  cudaGraphGetNodes(g, nodes.data(), &nn);
  for (auto nd : nodes) {
    size_t nd_out = 0;
    cudaGraphNodeGetDependentNodes(nd, nullptr, &nd_out);
    if (nd_out == 0) leaves.push_back(nd);
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  e = cudaGraphAddNode(&cnode, g, leaves.data(), leaves.size(), &cp);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_last_error("cudaGraphAddNode(while)", e);
    return MLSH_ERR_CUDA;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  auto capture = [&](cudaGraph_t into, StepFn fn, const SolveCtx &cc) {
    cudaError_t ce = cudaStreamBeginCaptureToGraph(h.capture_stream, into, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      cudaError_t e2 = fn(cc, h.capture_stream, cr);
      cudaGraph_t bb = nullptr;
      ce = cudaStreamEndCapture(h.capture_stream, &bb);
      if (ce == cudaSuccess) ce = e2;
    }
    return ce;
  };
  if (c.kind == kMixedBiCGSTAB) {
    // body = one FP32 iteration, then IF (update pending) { reliable update }
    cudaGraphConditionalHandle hif;
    e = cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault);
    SolveCtx c2 = c;
    c2.upd_cond = CondRef{hif, 1};
    if (e == cudaSuccess) e = capture(body, mixbi_main, c2);
    if (e == cudaSuccess) {
      size_t bn = 0;
      cudaGraphGetNodes(body, nullptr, &bn);
      std::vector<cudaGraphNode_t> bnodes(bn), bleaves;
      cudaGraphGetNodes(body, bnodes.data(), &bn);
      for (auto nd : bnodes) {
        size_t nd_out = 0;
        cudaGraphNodeGetDependentNodes(nd, nullptr, &nd_out);
        if (nd_out == 0) bleaves.push_back(nd);
      }
      cudaGraphNodeParams ip = {};
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = hif;
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      cudaGraphNode_t inode;
      e = cudaGraphAddNode(&inode, body, bleaves.data(), bleaves.size(), &ip);
      if (e == cudaSuccess) e = capture(ip.conditional.phGraph_out[0], mixbi_update, c2);
    }
  } else {
    e = capture(body, iter, c);
  }
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_last_error("capture solver body", e);
    return MLSH_ERR_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    set_last_error("cudaGraphInstantiate", e);
    return MLSH_ERR_CUDA;
  }
  out.graph = g;
  out.exec = ex;
  return MLSH_SUCCESS;
}

int get_graph(const SolveCtx &c, Handle &h, cudaGraphExec_t *ex) {
  GraphCache &gc = cache_of(h);
  ++gc.clock;
  for (auto &e : gc.entries) {
    if (e.kind == c.kind && e.dtype == c.dtype && e.jac == c.jac && e.plan == c.plan &&
        e.b == c.b && e.x == c.x && e.d == c.d && e.ws == c.ws && e.n == c.n &&
        e.pc == c.pc) {
      e.last_use = gc.clock;
      *ex = e.exec;
      return MLSH_SUCCESS;
    }
  }
  GraphEntry ne{c.kind, c.dtype, c.jac, c.plan, c.b, c.x, c.d, c.ws, c.n, nullptr, nullptr,
                gc.clock, c.pc};
  int st = build_graph(c, h, ne);
  if (st != MLSH_SUCCESS) return st;
  constexpr size_t kMaxEntries = 16;
  if (gc.entries.size() >= kMaxEntries) {
    size_t victim = 0;
    for (size_t i = 1; i < gc.entries.size(); ++i)
      if (gc.entries[i].last_use < gc.entries[victim].last_use) victim = i;
    destroy_entry(gc.entries[victim]);
    gc.entries.erase(gc.entries.begin() + victim);
  }
  gc.entries.push_back(ne);
  *ex = ne.exec;
  return MLSH_SUCCESS;
}

void purge_graphs(Handle &h, const CsrPlan *plan, const void *ws) {
  if (!h.graph_cache) return;
  GraphCache &gc = cache_of(h);
  for (size_t i = 0; i < gc.entries.size();) {
    if ((plan && gc.entries[i].plan == plan) || (ws && gc.entries[i].ws == ws)) {
      destroy_entry(gc.entries[i]);
      gc.entries.erase(gc.entries.begin() + i);
    } else {
      ++i;
    }
  }
}

int ensure_ws(Handle &h, size_t bytes) {
  if (h.ws_bytes >= bytes) return MLSH_SUCCESS;
  if (h.ws) {
    cudaStreamSynchronize(h.stream);
    purge_graphs(h, nullptr, h.ws);
    pool_free(h.ws, h.stream);
    h.ws = nullptr;
    h.ws_bytes = 0;
  }
  if (pool_alloc(&h.ws, bytes, h.stream) != cudaSuccess) {
    cudaGetLastError();
    return MLSH_ERR_OOM;
  }
  h.ws_bytes = bytes;
  return MLSH_SUCCESS;
}

// One system on the cluster engine.  Returns MLSH_NOT_IMPL when the system
// does not fit it (the caller then uses the kernel engine).
int cluster_solve_one(Kind kind, Handle &h, CsrPlan &p, const void *b, void *x,
                      const mlsh_solver_opts *opts, mlsh_solver_result *res) {
  const int64_t n = p.n_rows;
  const int rpc = cluster_rows_for(kind == kCG ? 0 : 1, p.dtype, n, opts->cluster_rows);
  if (rpc == 0) return MLSH_NOT_IMPL;
  const int csize = (int)((n + rpc - 1) / rpc);
  const bool jac = opts->precond == MLSH_PRECOND_JACOBI;
  const size_t esz = (size_t)dtype_size(p.dtype);
  const size_t vec = ((size_t)n * esz + 255) / 256 * 256;
  // workspace: [system record][queue][inverse diagonal][r0]
  int st = ensure_ws(h, 512 + 2 * vec);
  if (st != MLSH_SUCCESS) return st;
  char *ws = static_cast<char *>(h.ws);
  ClusterSystem *d_sys = reinterpret_cast<ClusterSystem *>(ws);
  unsigned *d_queue = reinterpret_cast<unsigned *>(ws + 256);
  const bool want_hist = opts->history != nullptr && opts->history_len > 0;
  if (want_hist && h.hist_cap < opts->history_len) {
    pool_free(h.hist, h.stream);
    h.hist = nullptr;
    h.hist_cap = 0;
    if (pool_alloc(&h.hist, sizeof(double) * (size_t)opts->history_len, h.stream) !=
        cudaSuccess) {
      cudaGetLastError();
      return MLSH_ERR_OOM;
    }
    h.hist_cap = opts->history_len;
  }
  ClusterSystem *hs = static_cast<ClusterSystem *>(h.host_cluster);
  std::memset(hs, 0, sizeof(ClusterSystem));
  hs->rp = p.row_ptr;
  hs->ci = p.col_ind;
  hs->val = p.val;
  hs->b = b;
  hs->x = x;
  hs->dinv = ws + 512;
  hs->aux = ws + 512 + vec;
  hs->n = (int)n;
  hs->tol = opts->tol;
  hs->maxiter = opts->maxiter;
  hs->miniter = opts->miniter;
  hs->hist = want_hist ? h.hist : nullptr;
  hs->hist_cap = want_hist ? opts->history_len : 0;
  hs->status = kRunning;
  MLSH_CUDA_TRY(cudaMemcpyAsync(d_sys, hs, sizeof(ClusterSystem), cudaMemcpyHostToDevice,
                                h.stream));
  MLSH_CUDA_TRY(cudaMemsetAsync(d_queue, 0, sizeof(unsigned), h.stream));
  st = cluster_launch(h, kind == kCG ? 0 : 1, p.dtype, jac, d_sys, 1, d_queue, rpc, csize, 1,
                      cluster_budget(opts), h.stream);
  if (st != MLSH_SUCCESS) return st;
  MLSH_CUDA_TRY(cudaMemcpyAsync(hs, d_sys, sizeof(ClusterSystem), cudaMemcpyDeviceToHost,
                                h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  res->status = hs->status;
  res->iters = hs->iters;
  res->final_resid = hs->resid;
  if (want_hist) {
    const int64_t k = std::min<int64_t>(hs->iters, opts->history_len);
    if (k > 0)
      MLSH_CUDA_TRY(cudaMemcpy(opts->history, h.hist, sizeof(double) * (size_t)k,
                               cudaMemcpyDeviceToHost));
  }
  return res->status;
}

int solve_common(Kind kind, mlsh_handle hs, mlsh_csr_plan ps, const void *b, void *x,
                 const mlsh_solver_opts *opts, mlsh_solver_result *res,
                 const Precond *pc = nullptr) {
  if (!hs || !ps || !opts) return MLSH_ERR_INVALID_ARG;
  Handle &h = hs->h;
  CsrPlan &p = ps->p;
  if (p.n_rows != p.n_cols) {
    if (res) res->status = MLSH_SOLVER_SIZE_ERROR;
    return MLSH_SOLVER_SIZE_ERROR;
  }
  if (!pc && opts->precond != MLSH_PRECOND_NONE && opts->precond != MLSH_PRECOND_JACOBI)
    return MLSH_ERR_INVALID_ARG;
  const int64_t n = p.n_rows;
  if (pc && pc->n != n) return MLSH_ERR_INVALID_ARG;
  if (n > 0 && (!b || !x)) return MLSH_ERR_INVALID_ARG;
  mlsh_solver_result local{};
  if (!res) res = &local;
  if (n == 0 && kind == kSOR) {
    // ||b|| = 0: the relative residual is 0 * inf = NaN at the first check
    res->final_resid = 0.0;
    res->iters = opts->maxiter > 0 ? 1 : 0;
    res->status = opts->maxiter > 0 ? MLSH_SOLVER_RESIDUAL_NAN : MLSH_SOLVER_MAXITER;
    return res->status;
  }
  if (n == 0) {
    // nothing to solve: ||r|| = 0 < tol from the first iteration on, so the
    // loop ends at max(1, miniter) unless maxiter comes first or tol <= 0
    const int64_t need = std::max<int64_t>(1, opts->miniter);
    res->final_resid = 0.0;
    if (0.0 < opts->tol && need <= opts->maxiter) {
      res->iters = need;
      res->status = MLSH_SUCCESS;
    } else {
      res->iters = std::max<int64_t>(0, opts->maxiter);
      res->status = MLSH_SOLVER_MAXITER;
    }
    return res->status;
  }
  if (!pc && (opts->engine == MLSH_ENGINE_CLUSTER ||
              (opts->engine == MLSH_ENGINE_AUTO && opts->maxiter <= kClusterMaxIterAuto))) {
    const int st = cluster_solve_one(kind, h, p, b, x, opts, res);
    if (st != MLSH_NOT_IMPL) return st;
    if (opts->engine == MLSH_ENGINE_CLUSTER) return MLSH_ERR_INVALID_ARG;
  }
  if (pc) {
    // the sweeps' poll bound is a launch parameter: graphs that captured
    // another one are dropped
    const unsigned polls =
        opts->wait_polls > 0 ? (unsigned)std::min<int64_t>(opts->wait_polls, 1u << 30)
                             : kDefaultWaitPolls;
    if (pc->wait_polls != polls) {
      purge_precond_graphs(h, pc);
      const_cast<Precond *>(pc)->wait_polls = polls;
    }
  }
  SolveCtx c;
  c.kind = kind;
  c.dtype = p.dtype;
  c.jac = !pc && opts->precond == MLSH_PRECOND_JACOBI;
  c.pc = pc;
  c.plan = &p;
  c.h = &h;
  c.b = b;
  c.x = x;
  c.d = nullptr;
  c.n = n;
  c.stride = n;
  if (c.jac) {
    int st = plan_inv_diag(p, h.stream, &c.d);
    if (st != MLSH_SUCCESS) return st;
  }
  const int nvec = kind == kSOR ? 2 : (kind == kCG ? (pc ? 4 : 3) : 8);
  const size_t esz = (size_t)dtype_size(p.dtype);
  // round each vector up to 256 bytes so every work vector stays aligned
  const int64_t n_al = (int64_t)(((size_t)n * esz + 255) / 256 * 256 / esz);
  int st = ensure_ws(h, (size_t)nvec * (size_t)n_al * esz);
  if (st != MLSH_SUCCESS) return st;
  c.ws = h.ws;
  c.stride = n_al;

  // configuration + fresh iteration state
  SolverState *hst = h.host_state;
  std::memset(hst, 0, sizeof(SolverState));
  hst->tol = opts->tol;
  hst->maxiter = opts->maxiter;
  hst->miniter = opts->miniter;
  hst->status = kRunning;
  hst->done = 0;
  const bool want_hist = opts->history != nullptr && opts->history_len > 0;
  if (want_hist) {
    if (h.hist_cap < opts->history_len) {
      pool_free(h.hist, h.stream);
      h.hist = nullptr;
      h.hist_cap = 0;
      if (pool_alloc(&h.hist, sizeof(double) * (size_t)opts->history_len, h.stream) !=
          cudaSuccess) {
        cudaGetLastError();
        h.hist = nullptr;
        return MLSH_ERR_OOM;
      }
      h.hist_cap = opts->history_len;
    }
    hst->hist = h.hist;
    hst->hist_cap = opts->history_len;
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(h.state, hst, sizeof(SolverState), cudaMemcpyHostToDevice,
                                h.stream));
  MLSH_CUDA_TRY(cudaMemsetAsync(h.err_flag, 0, sizeof(int), h.stream));

  bool graph_ok = false;
  if (opts->use_graph) {
    cudaGraphExec_t ex = nullptr;
    if (get_graph(c, h, &ex) == MLSH_SUCCESS) {
      MLSH_CUDA_TRY(cudaGraphLaunch(ex, h.stream));
      graph_ok = true;
    } else {
      cudaGetLastError();
    }
  }
  if (!graph_ok) {
    StepFn init, iter;
    pick_steps(c, &init, &iter);
    CondRef none{0, 0};
    MLSH_CUDA_TRY(init(c, h.stream, none));
    const int every = opts->check_every > 0 ? opts->check_every : 16;
    while (true) {
      for (int k = 0; k < every; ++k) MLSH_CUDA_TRY(iter(c, h.stream, none));
      MLSH_CUDA_TRY(cudaMemcpyAsync(hst, h.state, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                    h.stream));
      MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
      if (hst->done) break;
    }
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(hst, h.state, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                h.stream));
  int err = 0;
  MLSH_CUDA_TRY(cudaMemcpyAsync(&h.host_scalars[7], h.err_flag, sizeof(int),
                                cudaMemcpyDeviceToHost, h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  std::memcpy(&err, &h.host_scalars[7], sizeof(int));
  if (err != 0) return err;
  res->status = hst->status;
  res->iters = hst->iter;
  res->final_resid = hst->resid;
  if (want_hist) {
    const int64_t k = std::min<int64_t>(hst->iter, opts->history_len);
    if (k > 0)
      MLSH_CUDA_TRY(cudaMemcpy(opts->history, h.hist, sizeof(double) * (size_t)k,
                               cudaMemcpyDeviceToHost));
  }
  return res->status;
}

}  // namespace

// Mixed-precision BiCGSTAB with reliable updates on the kernel engine (see
// MixInitBody): p is the FP64 matrix, p32 its FP32 copy, r64 an n-vector.
int mixed_bicgstab_kernels(Handle &h, CsrPlan &p, CsrPlan &p32, double *r64,
                           const double *dinv64, const void *b, void *x,
                           const mlsh_solver_opts *opts, double inner_tol,
                           mlsh_solver_result *res) {
  const int64_t n = p.n_rows;
  SolveCtx c;
  c.kind = kMixedBiCGSTAB;
  c.dtype = MLSH_F32;
  c.jac = dinv64 != nullptr;
  c.plan = &p32;
  c.plan64 = &p;
  c.r64 = r64;
  c.h = &h;
  c.b = b;
  c.x = x;
  c.d = dinv64;
  c.n = n;
  const int64_t n_al = (int64_t)(((size_t)n * 4 + 255) / 256 * 256 / 4);
  int st = ensure_ws(h, (size_t)7 * (size_t)n_al * 4);
  if (st != MLSH_SUCCESS) return st;
  c.ws = h.ws;
  c.stride = n_al;

  SolverState *hst = h.host_state;
  std::memset(hst, 0, sizeof(SolverState));
  hst->tol = opts->tol;
  hst->maxiter = opts->maxiter;
  hst->miniter = opts->miniter;
  hst->delta = inner_tol;
  hst->status = kRunning;
  hst->done = 0;
  const bool want_hist = opts->history != nullptr && opts->history_len > 0;
  if (want_hist) {
    if (h.hist_cap < opts->history_len) {
      pool_free(h.hist, h.stream);
      h.hist = nullptr;
      h.hist_cap = 0;
      if (pool_alloc(&h.hist, sizeof(double) * (size_t)opts->history_len, h.stream) !=
          cudaSuccess) {
        cudaGetLastError();
        return MLSH_ERR_OOM;
      }
      h.hist_cap = opts->history_len;
    }
    hst->hist = h.hist;
    hst->hist_cap = opts->history_len;
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(h.state, hst, sizeof(SolverState), cudaMemcpyHostToDevice,
                                h.stream));
  MLSH_CUDA_TRY(cudaMemsetAsync(h.err_flag, 0, sizeof(int), h.stream));
  bool graph_ok = false;
  if (opts->use_graph) {
    cudaGraphExec_t ex = nullptr;
    if (get_graph(c, h, &ex) == MLSH_SUCCESS) {
      MLSH_CUDA_TRY(cudaGraphLaunch(ex, h.stream));
      graph_ok = true;
    } else {
      cudaGetLastError();
    }
  }
  if (!graph_ok) {
    StepFn init, iter;
    pick_steps(c, &init, &iter);
    CondRef none{0, 0};
    MLSH_CUDA_TRY(init(c, h.stream, none));
    const int every = opts->check_every > 0 ? opts->check_every : 16;
    while (true) {
      MLSH_CUDA_TRY(cudaMemcpyAsync(hst, h.state, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                    h.stream));
      MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
      if (hst->done) break;
      for (int k = 0; k < every; ++k) MLSH_CUDA_TRY(iter(c, h.stream, none));
    }
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(hst, h.state, sizeof(SolverState), cudaMemcpyDeviceToHost,
                                h.stream));
  MLSH_CUDA_TRY(cudaMemcpyAsync(&h.host_scalars[7], h.err_flag, sizeof(int),
                                cudaMemcpyDeviceToHost, h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  int err = 0;
  std::memcpy(&err, &h.host_scalars[7], sizeof(int));
  if (err != 0) return err;
  res->status = hst->status;
  res->iters = hst->iter;
  res->final_resid = hst->resid;
  res->outer_iters = (int)hst->outer;
  if (want_hist) {
    const int64_t k = std::min<int64_t>(hst->outer + 1, opts->history_len);
    if (k > 0)
      MLSH_CUDA_TRY(cudaMemcpy(opts->history, h.hist, sizeof(double) * (size_t)k,
                               cudaMemcpyDeviceToHost));
  }
  return res->status;
}

void release_solver_graphs(Handle &h) {
  if (h.graph_cache) {
    GraphCache &gc = cache_of(h);
    for (auto &e : gc.entries) destroy_entry(e);
    delete static_cast<GraphCache *>(h.graph_cache);
    h.graph_cache = nullptr;
  }
  cudaStreamSynchronize(h.stream);
  pool_free(h.ws, h.stream);
  h.ws = nullptr;
  h.ws_bytes = 0;
  pool_free(h.hist, h.stream);
  cudaStreamSynchronize(h.stream);
  h.hist = nullptr;
  h.hist_cap = 0;
}

void purge_precond_graphs(Handle &h, const Precond *pc) {
  if (!h.graph_cache || !pc) return;
  GraphCache &gc = cache_of(h);
  for (size_t i = 0; i < gc.entries.size();) {
    if (gc.entries[i].pc == pc) {
      destroy_entry(gc.entries[i]);
      gc.entries.erase(gc.entries.begin() + i);
    } else {
      ++i;
    }
  }
}

// The SOR solver's sweep (scaling omega / diag(A)) kept with the plan.
struct SorCache {
  Precond pc;
  double omega = 0.0;
};

void sor_cache_release(CsrPlan &p) {
  auto *c = static_cast<SorCache *>(p.sor);
  if (!c) return;
  if (p.handle) purge_precond_graphs(*p.handle, &c->pc);
  precond_release(c->pc);
  delete c;
  p.sor = nullptr;
}

int sor_cache_get(Handle &h, CsrPlan &p, double omega, const Precond **out) {
  auto *c = static_cast<SorCache *>(p.sor);
  if (c && c->omega == omega) {
    *out = &c->pc;
    return MLSH_SUCCESS;
  }
  sor_cache_release(p);
  c = new (std::nothrow) SorCache;
  if (!c) return MLSH_ERR_OOM;
  const int st = precond_build(h, p, MLSH_PRECOND_SOR, omega, true, c->pc);
  if (st != MLSH_SUCCESS) {
    delete c;
    return st;
  }
  c->omega = omega;
  p.sor = c;
  *out = &c->pc;
  return MLSH_SUCCESS;
}

void release_plan_extras(CsrPlan &p) {
  sor_cache_release(p);
  if (p.handle) purge_graphs(*p.handle, &p, nullptr);
  mixed_release(p);
  transpose_release(p);
}

void invalidate_plan_extras(CsrPlan &p) {
  sor_cache_release(p);
  if (p.handle) purge_graphs(*p.handle, &p, nullptr);
  mixed_invalidate(p);
  transpose_invalidate(p);
}

}  // namespace mlsh

using namespace mlsh;

extern "C" {

int mlsh_solver_opts_default(mlsh_solver_opts *o) {
  if (!o) return MLSH_ERR_INVALID_ARG;
  o->tol = 1.0e-8;
  o->maxiter = INT64_MAX;
  o->miniter = 0;
  o->precond = MLSH_PRECOND_JACOBI;
  o->use_graph = 1;
  o->check_every = 0;
  o->engine = MLSH_ENGINE_AUTO;
  o->history = nullptr;
  o->history_len = 0;
  o->cluster_rows = 0;
  o->reserved = 0;
  o->time_limit = 0.0;
  o->wait_polls = 0;
  return MLSH_SUCCESS;
}

int mlsh_cg_solve(mlsh_handle hs, mlsh_csr_plan ps, const void *b, void *x,
                  const mlsh_solver_opts *opts, mlsh_solver_result *res) {
  return solve_common(kCG, hs, ps, b, x, opts, res);
}

int mlsh_bicgstab_solve(mlsh_handle hs, mlsh_csr_plan ps, const void *b, void *x,
                        const mlsh_solver_opts *opts, mlsh_solver_result *res) {
  return solve_common(kBiCGSTAB, hs, ps, b, x, opts, res);
}

int mlsh_cg_solve_precond(mlsh_handle hs, mlsh_csr_plan ps, mlsh_precond pc, const void *b,
                          void *x, const mlsh_solver_opts *opts, mlsh_solver_result *res) {
  if (!pc) return MLSH_ERR_INVALID_ARG;
  return solve_common(kCG, hs, ps, b, x, opts, res, &pc->p);
}

int mlsh_bicgstab_solve_precond(mlsh_handle hs, mlsh_csr_plan ps, mlsh_precond pc,
                                const void *b, void *x, const mlsh_solver_opts *opts,
                                mlsh_solver_result *res) {
  if (!pc) return MLSH_ERR_INVALID_ARG;
  return solve_common(kBiCGSTAB, hs, ps, b, x, opts, res, &pc->p);
}

int mlsh_sor_solve(mlsh_handle hs, mlsh_csr_plan ps, const void *b, void *x, double omega,
                   const mlsh_solver_opts *opts, mlsh_solver_result *res) {
  if (!hs || !ps || !opts || !(omega == omega)) return MLSH_ERR_INVALID_ARG;
  if (opts->precond != MLSH_PRECOND_NONE) return MLSH_ERR_INVALID_ARG;
  CsrPlan &p = ps->p;
  if (p.n_rows != p.n_cols) {
    if (res) res->status = MLSH_SOLVER_SIZE_ERROR;
    return MLSH_SOLVER_SIZE_ERROR;
  }
  const Precond *pc = nullptr;
  const int st = sor_cache_get(hs->h, p, omega, &pc);
  if (st != MLSH_SUCCESS) return st;
  return solve_common(kSOR, hs, ps, b, x, opts, res, pc);
}

}  // extern "C"
