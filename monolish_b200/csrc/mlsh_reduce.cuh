// Deterministic reductions.  Every sum is formed in a fixed order that
// depends only on the launch geometry (which depends only on the sizes), so
// repeated calls give bit-identical results:
//   thread partial (fixed element sequence) -> warp xor-tree -> warps in
//   index order -> one partial per CTA -> the last CTA to finish (arrival
//   counter) sums the CTA partials in index order.
#pragma once
#include "mlsh_ptx.cuh"

namespace mlsh {

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum NR values over the `nthreads` threads (multiple of 32, ids
// 0..nthreads-1 relative to `base_tid`) that call this together with
// named barrier `bar`.  `red` holds nthreads/32*NR doubles.  The result is
// valid in relative thread 0 only.
template <int NR>
__device__ __forceinline__ void group_sum(double (&v)[NR], double *red,
                                          int rel_tid, int nthreads,
                                          int bar) {
  const int lane = rel_tid & 31, warp = rel_tid >> 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) red[warp * NR + k] = v[k];
  }
  named_sync(bar, nthreads);
  if (rel_tid == 0) {
    const int nw = nthreads >> 5;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[w * NR + k];
      v[k] = s;
    }
  }
  named_sync(bar, nthreads);
}

// Publish this CTA's NR sums (valid in relative thread 0) and find out
// whether this CTA is the last to arrive.  Uniform result over the group.
template <int NR>
__device__ __forceinline__ bool publish_partials(const double (&v)[NR],
                                                 double *partials,
                                                 unsigned *counter, int *s_flag,
                                                 int rel_tid, int nthreads,
                                                 int bar) {
  if (rel_tid == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) partials[blockIdx.x * NR + k] = v[k];
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    *s_flag = (prev == gridDim.x - 1) ? 1 : 0;
  }
  named_sync(bar, nthreads);
  const bool last = *s_flag != 0;
  if (last) __threadfence();
  return last;
}

// In the last CTA: sum the per-CTA partials (nblocks x NR) and `nextra`
// extra records (nextra x NR, stride `extra_stride` doubles) in fixed order.
// Result valid in relative thread 0.  Resets the arrival counter.
template <int NR>
__device__ __forceinline__ void reduce_partials(double (&out)[NR],
                                                const double *partials,
                                                int nblocks,
                                                const double *extra,
                                                int nextra, int extra_stride,
                                                unsigned *counter, double *red,
                                                int rel_tid, int nthreads,
                                                int bar) {
#pragma unroll
  for (int k = 0; k < NR; ++k) out[k] = 0.0;
  for (int b = rel_tid; b < nblocks; b += nthreads) {
#pragma unroll
    for (int k = 0; k < NR; ++k) out[k] += __ldcg(partials + b * NR + k);
  }
  for (int e = rel_tid; e < nextra; e += nthreads) {
#pragma unroll
    for (int k = 0; k < NR; ++k) out[k] += __ldcg(extra + e * extra_stride + k);
  }
  group_sum<NR>(out, red, rel_tid, nthreads, bar);
  if (rel_tid == 0) *counter = 0u;
}

}  // namespace mlsh
