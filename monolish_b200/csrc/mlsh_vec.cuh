// Elementwise / reduction kernels over device vectors (HBM-bound streams).
//
// One generic grid-stride kernel runs a small "body" functor per element;
// bodies that produce sums accumulate NR doubles per thread, and the last
// CTA to finish (arrival counter) reduces the per-CTA partials in fixed
// order and calls body.finish() with the totals -- which is where solvers
// update their device-side scalars and convergence state without a host
// round trip.  Grid geometry depends only on n, so sums are reproducible.
#pragma once
#include <type_traits>

#include "mlsh_internal.cuh"
#include "mlsh_reduce.cuh"

namespace mlsh {

struct RedArgs {
  double *partials;
  unsigned *counter;
  const int *done;  // optional: skip the launch when *done != 0
};

// NR: number of sums; FIN: call body.finish(sums) in the last CTA.
template <int NR, bool FIN, typename Body>
__global__ void __launch_bounds__(kVecThreads)
    vec_kernel(int64_t n, Body body, RedArgs ra) {
  pdl_wait();
  pdl_launch_dependents();
  if (ra.done != nullptr && *ra.done != 0) return;
  constexpr int NA = NR > 0 ? NR : 1;
  __shared__ double red[kVecThreads / 32 * NA];
  __shared__ int last_flag;
  body.prepare();
  double acc[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) acc[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    body(i, acc);
  if constexpr (NR > 0 || FIN) {
    group_sum<NA>(acc, red, threadIdx.x, kVecThreads, 0);
    if (publish_partials<NA>(acc, ra.partials, ra.counter, &last_flag, threadIdx.x,
                             kVecThreads, 0)) {
      double tot[NA];
      reduce_partials<NA>(tot, ra.partials, (int)gridDim.x, nullptr, 0, NA, ra.counter,
                          red, threadIdx.x, kVecThreads, 0);
      if (threadIdx.x == 0) body.finish(tot);
    }
  }
}

// --------------------------------------------------------- packed form --
// Bodies that provide `template <int W> step(i, acc)` over W consecutive
// elements (and a host-side aligned() check of their pointers) run with
// 16-byte vector loads and stores: 4 floats or 2 doubles per access, four
// or two times the bytes in flight per load instruction.
template <typename T, int W>
struct alignas(sizeof(T) * W) Pack {
  T v[W];
};
template <int W, typename T>
__device__ __forceinline__ Pack<T, W> ldp(const T *p, int64_t i) {
  return *reinterpret_cast<const Pack<T, W> *>(p + i);
}
template <int W, typename T>
__device__ __forceinline__ void stp(T *p, int64_t i, const Pack<T, W> &x) {
  *reinterpret_cast<Pack<T, W> *>(p + i) = x;
}
inline bool al16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

template <int NR, bool FIN, int W, typename Body>
__global__ void __launch_bounds__(kVecThreads)
    vec_pack_kernel(int64_t n, Body body, RedArgs ra) {
  pdl_wait();
  pdl_launch_dependents();
  if (ra.done != nullptr && *ra.done != 0) return;
  constexpr int NA = NR > 0 ? NR : 1;
  __shared__ double red[kVecThreads / 32 * NA];
  __shared__ int last_flag;
  body.prepare();
  double acc[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) acc[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t np = n / W;
  for (int64_t q = gt; q < np; q += stride) body.template step<W>(q * W, acc);
  for (int64_t i = np * W + gt; i < n; i += stride) body.template step<1>(i, acc);
  if constexpr (NR > 0 || FIN) {
    group_sum<NA>(acc, red, threadIdx.x, kVecThreads, 0);
    if (publish_partials<NA>(acc, ra.partials, ra.counter, &last_flag, threadIdx.x,
                             kVecThreads, 0)) {
      double tot[NA];
      reduce_partials<NA>(tot, ra.partials, (int)gridDim.x, nullptr, 0, NA, ra.counter,
                          red, threadIdx.x, kVecThreads, 0);
      if (threadIdx.x == 0) body.finish(tot);
    }
  }
}

template <typename B, typename = void>
struct has_step : std::false_type {};
template <typename B>
struct has_step<B, std::void_t<decltype(&B::aligned)>> : std::true_type {};

// ---------------------------------------------------------------- bodies --
struct NoPrep {
  __device__ void prepare() {}
  __device__ void finish(const double *) {}
};

template <typename T>
struct DotBody : NoPrep {
  const T *x;
  const T *y;
  double *out;
  __device__ void operator()(int64_t i, double *acc) const {
    acc[0] += (double)x[i] * (double)y[i];
  }
  __device__ void finish(const double *s) { *out = s[0]; }
};

template <typename T>
struct Nrm2Body : NoPrep {
  const T *x;
  double *out;
  __device__ void operator()(int64_t i, double *acc) const {
    const double v = (double)x[i];
    acc[0] += v * v;
  }
  __device__ void finish(const double *s) { *out = sqrt(s[0]); }
};

template <typename T>
struct AxpyBody : NoPrep {  // y = alpha*x + y
  T alpha;
  const T *x;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = alpha * x[i] + y[i]; }
};

template <typename T>
struct XpayBody : NoPrep {  // y = x + alpha*y
  T alpha;
  const T *x;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = x[i] + alpha * y[i]; }
};

template <typename T>
struct AxpyzBody : NoPrep {  // z = alpha*x + y
  T alpha;
  const T *x;
  const T *y;
  T *z;
  __device__ void operator()(int64_t i, double *) const { z[i] = alpha * x[i] + y[i]; }
};

template <typename T>
struct CopyBody : NoPrep {
  const T *x;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = x[i]; }
};

template <typename T>
struct SubBody : NoPrep {  // y = a - b
  const T *a;
  const T *b;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = a[i] - b[i]; }
};

template <typename T>
struct MulBody : NoPrep {  // y = a .* b
  const T *a;
  const T *b;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = a[i] * b[i]; }
};

template <typename T>
struct RecipBody : NoPrep {  // y = 1 ./ a
  const T *a;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = T(1) / a[i]; }
};

template <typename T>
struct FillBody : NoPrep {
  T value;
  T *y;
  __device__ void operator()(int64_t i, double *) const { y[i] = value; }
};

// Grid for an n-element stream on this device.
inline int vec_grid(int64_t n, int num_sms) {
  int64_t g = (n + (int64_t)kVecThreads * 4 - 1) / ((int64_t)kVecThreads * 4);
  const int64_t cap = (int64_t)num_sms * kMaxVecBlocksPerSm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace mlsh
