// SOR / IC(0) / ILU(0) on the device: pattern analysis, the two
// factorizations, the synchronization-free triangular sweeps and the C ABI
// of the preconditioner object.  The algorithms and the reference each one
// follows are described in mlsh_precond.cuh.
//
// Arithmetic is written with explicitly rounded operations (no fused
// multiply-add), so that values follow a sequential evaluation's order:
//   * the factorizations apply every update to an entry in the order of the
//     row-by-row (IKJ) algorithms, and sum the IC inner products in
//     ascending column order: bit-identical to a sequential factorization;
//   * the forward sweeps accumulate each row in ascending column order, as
//     src/equation/kernel/sor_kernel.hpp:50-58 does, and the backward sweeps
//     a row's entries outside its 32-row block in ascending order, then those
//     inside it in descending order (the order of the block's chain);
//   * blocks whose rows depend only on the adjacent row are resolved by an
//     affine scan instead of the chain: there the rounding differs from the
//     sequential recurrence's (by a few units in the last place).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "mlsh_core.cuh"
#include "mlsh_precond.cuh"
#include "mlsh_ptx.cuh"

namespace mlsh {
namespace {

constexpr int kSweepThreads = 256;
constexpr int kSweepWarps = kSweepThreads / 32;
constexpr unsigned kWaitPolls = kDefaultWaitPolls;  // factorizations' polls per wait
constexpr unsigned kFull = 0xffffffffu;

// ---- explicitly rounded arithmetic
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }

// Waits until *flag == want.  Gives up (recording MLSH_ERR_TIMEOUT) after
// `polls` polls (kWaitPolls unless the solve asked for fewer), or soon after
// another warp has recorded an error.  The
// loop is a bare acquire poll (no timer reads, no sleeps): measured on the
// sweeps, this keeps the hop from a publishing warp to its waiters about
// half as long as polls interleaved with sleeps or timer reads.
__device__ __noinline__ bool wait_flag(const unsigned *flag, unsigned want, int *err,
                                      unsigned polls) {
  for (unsigned it = 0; it < polls; ++it) {
    if (ld_acquire_gpu(flag) == want) return true;
    if ((it & 1023u) == 1023u && *(volatile int *)err != 0) return false;
  }
  atomicCAS(err, 0, MLSH_ERR_TIMEOUT);
  return false;
}

// ---------------------------------------------------------------------------
// Pattern analysis: lo_end / up_beg per row, sorted in-range columns, first
// missing diagonal.
__global__ void split_rows_kernel(const int *rp, const int *ci, int n, int *lo_end,
                                  int *up_beg, int *bad, unsigned long long *missing) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = rp[i], e = rp[i + 1];
  int lo = e, up = e, prev = -1;
  for (int j = b; j < e; ++j) {
    const int c = ci[j];
    if (c <= prev || c >= n) atomicExch(bad, 1);
    prev = c;
    if (lo == e && c >= i) lo = j;
    if (up == e && c > i) up = j;
  }
  lo_end[i] = lo;
  up_beg[i] = up;
  if (up == lo) atomicMin(missing, (unsigned long long)i);
}

// SOR multipliers: scale_i = 1 / (w * a_ii), w = omega (preconditioner,
// sor.cpp:29-32) or 1/omega rounded to T (the solver, sor.cpp:112-115).
template <typename T>
__global__ void sor_scale_kernel(const T *val, const int *lo_end, const int *up_beg, int n,
                                 T w, T *scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int d = lo_end[i];
  const T aii = up_beg[i] > d ? val[d] : T(0);
  scale[i] = div_rn(T(1), mul_rn(w, aii));
}

// ---------------------------------------------------------------------------
// The sweeps.
template <typename T>
struct SweepArgs {
  const int *rp;
  const int *ci;
  const T *val;
  const int *lo_end;
  const int *up_beg;
  const T *scale;
  const T *rhs;
  T *out;
  int n;
  unsigned nb;
  unsigned long long *ticket;
  unsigned *flags;
  const int *done;
  int *err;
  const int *order;
  const int *dep_off;
  const int *dep_ids;
  unsigned polls;  // polls per wait before giving up
};

template <int MODE, typename T>
__device__ __forceinline__ T fwd_finish(T acc, T fin) {
  if constexpr (MODE == kSorFwd) return mul_rn(acc, fin);
  else if constexpr (MODE == kDiagFwd) return div_rn(acc, fin);
  else return acc;
}

// Takes this warp's ticket; false if the warp has no block or the launch
// is to be skipped.  Every warp with a block takes exactly one ticket, so a
// launch consumes nb tickets and the epoch is ticket / nb + 1.
template <typename T>
__device__ __forceinline__ bool sweep_ticket(const SweepArgs<T> &a, int lane,
                                             unsigned long long *t) {
  const unsigned gw = blockIdx.x * kSweepWarps + (threadIdx.x >> 5);
  if (gw >= a.nb) return false;
  unsigned long long v = 0;
  if (lane == 0) v = atomicAdd(a.ticket, 1ull);
  *t = __shfl_sync(kFull, v, 0);
  return !(a.done != nullptr && *(volatile const int *)a.done != 0);
}

// The lanes' stores are ordered before lane 0's by the warp barrier, and
// lane 0's release store (cumulative) makes them visible, at GPU scope, to
// every warp that acquires the flag.
__device__ __forceinline__ void publish_block(unsigned *flag, unsigned epoch, int lane) {
  __syncwarp();
  if (lane == 0) st_release_gpu(flag, epoch);
}

// Schedule entries: block id, and a bit marking blocks whose rows depend
// inside the block only on the adjacent row (row - 1 lower, row + 1 upper).
constexpr unsigned kScanBit = 0x80000000u;
constexpr unsigned kBlockMask = 0x7fffffffu;

// x_k = al_k + be_k x_{k-1} (REV: x_{k+1}) over the 32 lanes, as a
// Kogge-Stone scan of affine maps over register shuffles (log2 32 = 5 steps
// instead of a 32-step chain).  A lane with be_k == 0 takes nothing from its
// neighbour, so a non-finite value there does not leak into it.
template <bool REV, typename S>
__device__ __forceinline__ S affine_scan(S al, S be, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const S al2 = REV ? __shfl_down_sync(kFull, al, d) : __shfl_up_sync(kFull, al, d);
    const S be2 = REV ? __shfl_down_sync(kFull, be, d) : __shfl_up_sync(kFull, be, d);
    const bool in = REV ? lane + d < 32 : lane >= d;
    if (in && be != S(0)) {
      al = al + be * al2;
      be = be * be2;
    }
  }
  return al;
}

// Lanes wait, in parallel, for the flags of the block's dependency blocks.
__device__ __forceinline__ void wait_deps(const int *dep_off, const int *dep_ids,
                                          const unsigned *flags, unsigned blk, unsigned epoch,
                                          int *err, int lane, unsigned polls) {
  const int d1 = dep_off[blk + 1];
  for (int d = dep_off[blk] + lane; d < d1; d += 32)
    wait_flag(flags + dep_ids[d], epoch, err, polls);
  __syncwarp();
}

constexpr int kPre = 4;  // out-of-block entries fetched ahead of the wait

// Where a sweep's solution vector lives while the sweep runs: in global
// memory (other warps' blocks, read through L2 after their flag) or, for the
// single-CTA form, in shared memory.
template <typename T>
struct GlobalX {
  T *out;
  __device__ T get(int c) const { return __ldcg(out + c); }
  __device__ void put(int r, T v) const { out[r] = v; }
};
template <typename T>
struct SharedX {
  T *xs;
  __device__ T get(int c) const { return xs[c]; }
  __device__ void put(int r, T v) const { xs[r] = v; }
};

// What a lane knows of its row before any solution value is needed: its
// range of entries, right-hand side, finishing factor and first entries.
template <typename T>
struct RowState {
  int j, e, jb, split;
  T acc, fin, rh;
  T a1v;  // upper sweep: the row's first upper entry (row + 1 in a scan block)
  int pc[kPre];
  T pv[kPre];
};

// Loading a row's state takes two dependent steps: the row's own arrays
// (stage 1), then what they point to (stage 2).
// RHS = false: the matrix-only state (the sweep records), acc left 0.
template <typename T, int MODE, bool RHS = true>
__device__ __forceinline__ void fwd_load1(const SweepArgs<T> &a, unsigned ov, int lane,
                                          RowState<T> &st) {
  const int row = (int)(ov & kBlockMask) * 32 + lane;
  st.acc = T(0);
  st.fin = T(1);
  st.j = 0;
  st.e = 0;
  st.split = 0;  // kDiagFwd: whether the diagonal is stored
  if (row < a.n) {
    st.j = a.rp[row];
    st.e = a.lo_end[row];
    if constexpr (RHS) st.acc = a.rhs[row];
    if constexpr (MODE == kSorFwd) st.fin = a.scale[row];
    if constexpr (MODE == kDiagFwd) st.split = a.up_beg[row] > st.e;
  }
}
template <typename T, int MODE>
__device__ __forceinline__ void fwd_load2(const SweepArgs<T> &a, RowState<T> &st) {
  if constexpr (MODE == kDiagFwd) st.fin = st.split ? a.val[st.e] : T(0);
#pragma unroll
  for (int u = 0; u < kPre; ++u) {
    st.pc[u] = st.j + u < st.e ? a.ci[st.j + u] : 0x7fffffff;
    st.pv[u] = st.j + u < st.e ? a.val[st.j + u] : T(0);
  }
}
template <typename T, int MODE>
__device__ __forceinline__ void fwd_load(const SweepArgs<T> &a, unsigned ov, int lane,
                                         RowState<T> &st) {
  fwd_load1<T, MODE>(a, ov, lane, st);
  fwd_load2<T, MODE>(a, st);
}

// One 32-row block of the lower sweep, from its loaded state: every value
// outside the block must be final when this runs.
template <typename T, int MODE, class XS>
__device__ __forceinline__ void fwd_finish_block(const SweepArgs<T> &a, unsigned ov, int lane,
                                                 const XS &X, const RowState<T> &st) {
  const int base = (int)(ov & kBlockMask) * 32;
  const int row = base + lane;
  const bool valid = row < a.n;
  T acc = st.acc;
  const T fin = st.fin;
  int j = st.j;
  const int e = st.e;
  // entries left of the block (a prefix of the row), ascending
  T xs[kPre];
#pragma unroll
  for (int u = 0; u < kPre; ++u) xs[u] = st.pc[u] < base ? X.get(st.pc[u]) : T(0);
#pragma unroll
  for (int u = 0; u < kPre; ++u)
    if (st.pc[u] < base) {
      acc = sub_rn(acc, mul_rn(st.pv[u], xs[u]));
      ++j;
    }
  if (st.pc[kPre - 1] < base) {
    for (; j < e; ++j) {
      const int c = a.ci[j];
      if (c >= base) break;
      acc = sub_rn(acc, mul_rn(a.val[j], X.get(c)));
    }
  }
  T xv = T(0);
  if (ov & kScanBit) {
    // the block's only in-block dependencies are row - 1 -> row: the
    // recurrence x_k = al_k + be_k x_{k-1} as a 5-step affine scan; the
    // (row, row - 1) entry is normally among the prefetched ones
    const int d = j - st.j;
    T a1 = T(0);
    if (d < kPre) {
#pragma unroll
      for (int u = 0; u < kPre; ++u)
        if (u == d) a1 = st.pv[u];
    } else if (j < e) {
      a1 = a.val[j];
    }
    T al, be;
    if constexpr (MODE == kSorFwd) {
      al = acc * fin;
      be = -(a1 * fin);
    } else if constexpr (MODE == kDiagFwd) {
      al = acc / fin;
      be = -(a1 / fin);
    } else {
      al = acc;
      be = -a1;
    }
    xv = affine_scan<false>(al, be, lane);
  } else {
    // entries inside the block, ascending: a 32-step chain; the next two
    // are kept in registers so the chain carries no memory latency
    int c0 = 64, c1 = 64;
    T v0 = T(0), v1 = T(0);
    if (j < e) {
      c0 = a.ci[j] - base;
      v0 = a.val[j];
    }
    if (j + 1 < e) {
      c1 = a.ci[j + 1] - base;
      v1 = a.val[j + 1];
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      if (lane == k) xv = fwd_finish<MODE>(acc, fin);
      const T xk = __shfl_sync(kFull, xv, k);
      if (c0 == k) {
        acc = sub_rn(acc, mul_rn(v0, xk));
        c0 = c1;
        v0 = v1;
        ++j;
        if (j + 1 < e) {
          c1 = a.ci[j + 1] - base;
          v1 = a.val[j + 1];
        } else {
          c1 = 64;
        }
      }
    }
  }
  if (valid) X.put(row, xv);
}

template <typename T, int MODE, bool RHS = true>
__device__ __forceinline__ void bwd_load1(const SweepArgs<T> &a, unsigned ov, int lane,
                                          RowState<T> &st) {
  const int row = (int)(ov & kBlockMask) * 32 + lane;
  st.acc = T(0);
  st.fin = T(1);
  st.rh = T(0);
  st.jb = 0;
  st.e = 0;
  st.j = -1;  // kDiagBwd: position of the diagonal, -1 if not stored
  st.split = 0;
  if (row < a.n) {
    st.jb = a.up_beg[row];
    st.e = a.rp[row + 1];
    if constexpr (RHS) st.rh = a.rhs[row];
    if constexpr (MODE == kSorBwd) {
      st.fin = a.scale[row];
    } else {
      st.acc = st.rh;
      const int d = a.lo_end[row];
      st.j = st.jb > d ? d : -1;
    }
  }
}
template <typename T, int MODE>
__device__ __forceinline__ void bwd_load2(const SweepArgs<T> &a, unsigned ov, RowState<T> &st) {
  const int base = (int)(ov & kBlockMask) * 32;
  if constexpr (MODE != kSorBwd) st.fin = st.j >= 0 ? a.val[st.j] : T(0);
  st.a1v = st.jb < st.e ? a.val[st.jb] : T(0);
  int split = st.jb;
  while (split < st.e && a.ci[split] < base + 32) ++split;
  st.split = split;
#pragma unroll
  for (int u = 0; u < kPre; ++u) {
    st.pc[u] = st.split + u < st.e ? a.ci[st.split + u] : -1;
    st.pv[u] = st.split + u < st.e ? a.val[st.split + u] : T(0);
  }
}
template <typename T, int MODE>
__device__ __forceinline__ void bwd_load(const SweepArgs<T> &a, unsigned ov, int lane,
                                         RowState<T> &st) {
  bwd_load1<T, MODE>(a, ov, lane, st);
  bwd_load2<T, MODE>(a, ov, st);
}

// One 32-row block of the upper sweep, from its loaded state.
template <typename T, int MODE, class XS>
__device__ __forceinline__ void bwd_finish_block(const SweepArgs<T> &a, unsigned ov, int lane,
                                                 const XS &X, const RowState<T> &st) {
  const int base = (int)(ov & kBlockMask) * 32;
  const int row = base + lane;
  const bool valid = row < a.n;
  // SOR accumulates in double ("auto tmp = 0.0", sor_kernel.hpp:61-66)
  T acc = st.acc;
  const T fin = st.fin, rh = st.rh;
  double sacc = 0.0;
  const int jb = st.jb, e = st.e, split = st.split;
  // entries right of the block (the row's suffix from split), ascending
  T xs[kPre];
#pragma unroll
  for (int u = 0; u < kPre; ++u) xs[u] = st.pc[u] >= 0 ? X.get(st.pc[u]) : T(0);
#pragma unroll
  for (int u = 0; u < kPre; ++u)
    if (st.pc[u] >= 0) {
      const T prod = mul_rn(st.pv[u], xs[u]);
      if constexpr (MODE == kSorBwd) sacc = __dadd_rn(sacc, (double)prod);
      else acc = sub_rn(acc, prod);
    }
  for (int j = split + kPre; j < e; ++j) {
    const T prod = mul_rn(a.val[j], X.get(a.ci[j]));
    if constexpr (MODE == kSorBwd) sacc = __dadd_rn(sacc, (double)prod);
    else acc = sub_rn(acc, prod);
  }
  T xv = T(0);
  if (ov & kScanBit) {
    // only row + 1 -> row inside the block: z_k = al_k + be_k z_{k+1}
    const T a1 = (split > jb) ? st.a1v : T(0);
    if constexpr (MODE == kSorBwd) {
      const double al = (double)rh - sacc * (double)fin;
      const double be = -((double)a1 * (double)fin);
      xv = (T)affine_scan<true>(al, be, lane);
    } else {
      xv = affine_scan<true>(acc / fin, -(a1 / fin), lane);
    }
  } else {
    // entries inside the block, consumed from the highest column down
    int q = split - 1;
    int c0 = 64, c1 = 64;
    T v0 = T(0), v1 = T(0);
    if (q >= jb) {
      c0 = a.ci[q] - base;
      v0 = a.val[q];
    }
    if (q - 1 >= jb) {
      c1 = a.ci[q - 1] - base;
      v1 = a.val[q - 1];
    }
#pragma unroll
    for (int k = 31; k >= 0; --k) {
      if (lane == k) {
        if constexpr (MODE == kSorBwd)
          xv = (T)__dsub_rn((double)rh, __dmul_rn(sacc, (double)fin));
        else
          xv = div_rn(acc, fin);
      }
      const T xk = __shfl_sync(kFull, xv, k);
      if (c0 == k) {
        const T prod = mul_rn(v0, xk);
        if constexpr (MODE == kSorBwd) sacc = __dadd_rn(sacc, (double)prod);
        else acc = sub_rn(acc, prod);
        c0 = c1;
        v0 = v1;
        --q;
        if (q - 1 >= jb) {
          c1 = a.ci[q - 1] - base;
          v1 = a.val[q - 1];
        } else {
          c1 = 64;
        }
      }
    }
  }
  if (valid) X.put(row, xv);
}

// The multi-CTA sweep: one warp per block, blocks by ticket in level order,
// per-block flags between warps.
template <typename T, int MODE, bool BWD>
__global__ void __launch_bounds__(kSweepThreads) sweep_kernel(SweepArgs<T> a) {
  const int lane = threadIdx.x & 31;
  unsigned long long t;
  if (!sweep_ticket(a, lane, &t)) return;
  const unsigned epoch = (unsigned)(t / a.nb) + 1u;
  const unsigned ov = (unsigned)a.order[t % a.nb];
  const unsigned blk = ov & kBlockMask;
  RowState<T> st;
  if constexpr (BWD) bwd_load<T, MODE>(a, ov, lane, st);
  else fwd_load<T, MODE>(a, ov, lane, st);
  wait_deps(a.dep_off, a.dep_ids, a.flags, blk, epoch, a.err, lane, a.polls);
  if constexpr (BWD) bwd_finish_block<T, MODE>(a, ov, lane, GlobalX<T>{a.out}, st);
  else fwd_finish_block<T, MODE>(a, ov, lane, GlobalX<T>{a.out}, st);
  publish_block(a.flags + blk, epoch, lane);
}

// The single-CTA sweep for systems whose solution fits in shared memory:
// the CTA's warps take each level's blocks, a barrier separates the levels,
// the solution lives in shared memory and is written out at the end.
constexpr int kCtaThreads = 512;
constexpr size_t kCtaSweepBytes = 200 * 1024;

template <typename T>
__host__ __device__ inline size_t cta_x_bytes(int n) {
  return ((size_t)n * sizeof(T) + 15) / 16 * 16;
}
// shared memory of the single-CTA sweep: solution, schedule, level starts
template <typename T>
inline size_t cta_smem_bytes(int n, unsigned nb, int levels) {
  return cta_x_bytes<T>(n) + sizeof(int) * ((size_t)nb + (size_t)levels + 1);
}

template <typename T, int MODE, bool BWD>
__global__ void __launch_bounds__(kCtaThreads, 1)
    sweep_cta_kernel(SweepArgs<T> a, const int *level_off, int levels) {
  extern __shared__ __align__(16) unsigned char sweep_smem[];
  if (a.done != nullptr && *(volatile const int *)a.done != 0) return;
  // [solution: n T][schedule: nb block entries][level starts: levels + 1]
  T *xs = reinterpret_cast<T *>(sweep_smem);
  int *s_order = reinterpret_cast<int *>(sweep_smem + cta_x_bytes<T>(a.n));
  int *s_loff = s_order + a.nb;
  for (int i = threadIdx.x; i < (int)a.nb; i += blockDim.x) s_order[i] = a.order[i];
  for (int i = threadIdx.x; i <= levels; i += blockDim.x) s_loff[i] = level_off[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const SharedX<T> X{xs};
  // A software pipeline over the levels: while a level runs, each warp
  // holds its first block of the next two levels fully loaded and the row
  // arrays of its first block three levels ahead, so the two dependent
  // loads of a row's state overlap two to three levels' work and barriers
  // (the loads read only the matrix and the sweep's right-hand side, which
  // no level writes).
  auto load1 = [&](unsigned o, RowState<T> &st) {
    if constexpr (BWD) bwd_load1<T, MODE>(a, o, lane, st);
    else fwd_load1<T, MODE>(a, o, lane, st);
  };
  auto load2 = [&](unsigned o, RowState<T> &st) {
    if constexpr (BWD) bwd_load2<T, MODE>(a, o, st);
    else fwd_load2<T, MODE>(a, st);
  };
  // this warp's first block of level lv, if it has one
  auto first_of = [&](int lv, unsigned &ov) -> bool {
    if (lv >= levels || s_loff[lv] + warp >= s_loff[lv + 1]) return false;
    ov = (unsigned)s_order[s_loff[lv] + warp];
    return true;
  };
  RowState<T> cur, nxt, nn;
  unsigned ov_cur = 0, ov_nxt = 0, ov_nn = 0;
  const bool have0 = first_of(0, ov_cur);
  if (have0) {
    load1(ov_cur, cur);
    load2(ov_cur, cur);
  }
  bool have_cur = have0;
  bool have_nxt = first_of(1, ov_nxt);
  if (have_nxt) {
    load1(ov_nxt, nxt);
    load2(ov_nxt, nxt);
  }
  bool have_nn = first_of(2, ov_nn);
  if (have_nn) load1(ov_nn, nn);
  for (int lv = 0; lv < levels; ++lv) {
    const int q1 = s_loff[lv + 1];
    for (int q = s_loff[lv] + warp; q < q1; q += nw) {
      RowState<T> st;
      unsigned ov;
      if (q == s_loff[lv] + warp && have_cur) {
        st = cur;
        ov = ov_cur;
      } else {
        ov = (unsigned)s_order[q];
        load1(ov, st);
        load2(ov, st);
      }
      if constexpr (BWD) bwd_finish_block<T, MODE>(a, ov, lane, X, st);
      else fwd_finish_block<T, MODE>(a, ov, lane, X, st);
    }
    // advance: the next level's block is ready, the one after it gets its
    // second stage, the block three levels ahead its first
    have_cur = have_nxt;
    if (have_nxt) {
      cur = nxt;
      ov_cur = ov_nxt;
    }
    have_nxt = have_nn;
    if (have_nn) {
      nxt = nn;
      ov_nxt = ov_nn;
      load2(ov_nxt, nxt);
    }
    have_nn = first_of(lv + 3, ov_nn);
    if (have_nn) load1(ov_nn, nn);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) a.out[i] = xs[i];
}

// ---------------------------------------------------------------------------
// The single-CTA ring sweep.  What a block's lanes load before any solution
// value is needed depends on the matrix only, so it is computed once, when
// the preconditioner is built, into one record per block in level order:
//   [block entry (id | scan bit), 12 bytes pad]
//   [T: first entries' values (kPre x 32), finishing factor, a1v (32 each)]
//   [int: first entries' columns (kPre x 32), j, e, jb, split (32 each)]
// During a sweep a producer warp streams the records into a ring of slots in
// shared memory by 1-D bulk copies, up to `ring` blocks ahead of the level
// being solved (slots free once their level has passed the level barrier),
// and the right-hand side is bulk-copied into the shared solution vector at
// the start: each row reads its own right-hand side there before its block
// writes the row's solution over it (no other block reads an unsolved row).
// So a level's critical path holds shared-memory reads, the block's
// arithmetic and the barrier, and no global-memory latency.
template <typename T>
struct SweepRec {
  static constexpr int kHead = 16;
  static constexpr int kTBytes = (kPre + 2) * 32 * (int)sizeof(T);
  static constexpr int kIntBytes = (kPre + 4) * 32 * 4;
  static constexpr int kBytes = kHead + kTBytes + kIntBytes;
  static_assert(kBytes % 16 == 0, "records are copied in 16-byte units");
  __device__ static const T *tv(const unsigned char *r) {
    return reinterpret_cast<const T *>(r + kHead);
  }
  __device__ static const int *iv(const unsigned char *r) {
    return reinterpret_cast<const int *>(r + kHead + kTBytes);
  }
};

template <typename T, int MODE, bool BWD>
__global__ void __launch_bounds__(kSweepThreads)
    sweep_rec_kernel(SweepArgs<T> a, unsigned char *rec) {
  const unsigned q = blockIdx.x * kSweepWarps + (threadIdx.x >> 5);
  if (q >= a.nb) return;
  const int lane = threadIdx.x & 31;
  const unsigned ov = (unsigned)a.order[q];
  RowState<T> st{};
  if constexpr (BWD) {
    bwd_load1<T, MODE, false>(a, ov, lane, st);
    bwd_load2<T, MODE>(a, ov, st);
  } else {
    fwd_load1<T, MODE, false>(a, ov, lane, st);
    fwd_load2<T, MODE>(a, st);
  }
  unsigned char *r = rec + (size_t)q * SweepRec<T>::kBytes;
  T *tv = reinterpret_cast<T *>(r + SweepRec<T>::kHead);
  int *iv = reinterpret_cast<int *>(r + SweepRec<T>::kHead + SweepRec<T>::kTBytes);
  if (lane < 4) reinterpret_cast<unsigned *>(r)[lane] = lane == 0 ? ov : 0u;
#pragma unroll
  for (int u = 0; u < kPre; ++u) {
    tv[u * 32 + lane] = st.pv[u];
    iv[u * 32 + lane] = st.pc[u];
  }
  tv[kPre * 32 + lane] = st.fin;
  tv[(kPre + 1) * 32 + lane] = st.a1v;
  iv[kPre * 32 + lane] = st.j;
  iv[(kPre + 1) * 32 + lane] = st.e;
  iv[(kPre + 2) * 32 + lane] = st.jb;
  iv[(kPre + 3) * 32 + lane] = st.split;
}

constexpr int kRingMaxSlots = 64;
constexpr int kRingMinSlots = 8;
constexpr size_t kRingSweepBytes = 225 * 1024;

// shared memory of the ring sweep: solution, level starts, ring, barriers
template <typename T>
inline size_t ring_smem_bytes(int n, int levels, int slots) {
  const size_t loff = ((size_t)(levels + 1) * sizeof(int) + 15) / 16 * 16;
  return cta_x_bytes<T>(n) + loff + (size_t)slots * SweepRec<T>::kBytes +
         ((size_t)slots + 2) * 8;
}

// Waits for a ring barrier phase, at most `polls` polls.
__device__ __forceinline__ bool ring_wait(uint32_t bar, uint32_t parity, unsigned polls) {
  for (unsigned it = 0; it < polls; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

template <typename T, int MODE, bool BWD>
__global__ void __launch_bounds__(kCtaThreads, 1)
    sweep_ring_kernel(SweepArgs<T> a, const int *level_off, int levels,
                      const unsigned char *rec, int slots) {
  extern __shared__ __align__(16) unsigned char sweep_smem[];
  if (a.done != nullptr && *(volatile const int *)a.done != 0) return;
  constexpr int kRec = SweepRec<T>::kBytes;
  const size_t xb = cta_x_bytes<T>(a.n);
  const size_t lb = ((size_t)(levels + 1) * sizeof(int) + 15) / 16 * 16;
  T *xs = reinterpret_cast<T *>(sweep_smem);
  int *s_loff = reinterpret_cast<int *>(sweep_smem + xb);
  unsigned char *ring = sweep_smem + xb + lb;
  uint64_t *bars = reinterpret_cast<uint64_t *>(ring + (size_t)slots * kRec);
  // bars[0, slots): one per ring slot; bars[slots]: the right-hand side;
  // bars[slots + 1] (as an int): set when a wait gave up
  int *s_fail = reinterpret_cast<int *>(bars + slots + 1);
  const uint32_t bar0 = smem_addr(bars);
  const uint32_t bar_rhs = bar0 + 8u * (uint32_t)slots;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kCtaThreads / 32;
  const int nw = kWarps - 1;  // the last warp produces
  const bool producer = warp == kWarps - 1;
  const int shift = 31 - __clz(slots);  // slots is a power of two
  for (int i = threadIdx.x; i <= levels; i += blockDim.x) s_loff[i] = level_off[i];
  // the right-hand side's bulk-copyable part: 16-byte aligned, whole chunks
  const bool rhs_bulk = (reinterpret_cast<uintptr_t>(a.rhs) & 15u) == 0;
  const uint32_t rhs_bytes = rhs_bulk ? (uint32_t)((size_t)a.n * sizeof(T) / 16 * 16) : 0u;
  if (threadIdx.x == 0) {
    for (int k = 0; k < slots + 1; ++k) mbar_init(bar0 + 8u * (uint32_t)k, 1);
    *s_fail = 0;
    fence_mbar_init();
  }
  __syncthreads();
  int issued = 0;  // producer lane 0: records copied so far
  if (producer && lane == 0 && rhs_bytes > 0) {
    mbar_arrive_expect_tx(bar_rhs, rhs_bytes);
    bulk_g2s(smem_addr(xs), a.rhs, rhs_bytes, bar_rhs);
  }
  // what the bulk copy does not cover, by plain loads
  for (int i = (int)(rhs_bytes / sizeof(T)) + (int)threadIdx.x; i < a.n; i += blockDim.x)
    xs[i] = a.rhs[i];
  if (rhs_bytes > 0 && !ring_wait(bar_rhs, 0, a.polls)) *s_fail = 1;
  __syncthreads();
  const SharedX<T> X{xs};
  for (int lv = 0; lv < levels; ++lv) {
    const int q0 = s_loff[lv], q1 = s_loff[lv + 1];
    if (producer) {
      if (lane == 0 && *s_fail == 0) {
        // slots of blocks below q0 are free: their level has passed the
        // barrier (after a failed wait nothing more is issued, so every slot
        // has at most one copy in flight)
        const int lim = min((int)a.nb, q0 + slots);
        if (issued < lim) fence_proxy_async_smem();
        for (; issued < lim; ++issued) {
          const int slot = issued & (slots - 1);
          const uint32_t bar = bar0 + 8u * (uint32_t)slot;
          mbar_arrive_expect_tx(bar, (uint32_t)kRec);
          bulk_g2s(smem_addr(ring + (size_t)slot * kRec), rec + (size_t)issued * kRec,
                   (uint32_t)kRec, bar);
        }
      }
    } else {
      for (int q = q0 + warp; q < q1; q += nw) {
        if (*(volatile int *)s_fail) break;
        const int slot = q & (slots - 1);
        if (!ring_wait(bar0 + 8u * (uint32_t)slot, (uint32_t)(q >> shift) & 1u, a.polls)) {
          *s_fail = 1;
          break;
        }
        const unsigned char *r = ring + (size_t)slot * kRec;
        const T *tv = SweepRec<T>::tv(r);
        const int *iv = SweepRec<T>::iv(r);
        const unsigned ov = *reinterpret_cast<const unsigned *>(r);
        RowState<T> st;
#pragma unroll
        for (int u = 0; u < kPre; ++u) {
          st.pv[u] = tv[u * 32 + lane];
          st.pc[u] = iv[u * 32 + lane];
        }
        st.fin = tv[kPre * 32 + lane];
        st.a1v = tv[(kPre + 1) * 32 + lane];
        st.j = iv[kPre * 32 + lane];
        st.e = iv[(kPre + 1) * 32 + lane];
        st.jb = iv[(kPre + 2) * 32 + lane];
        st.split = iv[(kPre + 3) * 32 + lane];
        const int row = (int)(ov & kBlockMask) * 32 + lane;
        const T own = row < a.n ? xs[row] : T(0);
        if constexpr (BWD) {
          st.rh = own;
          st.acc = MODE == kSorBwd ? T(0) : own;
          bwd_finish_block<T, MODE>(a, ov, lane, X, st);
        } else {
          st.acc = own;
          fwd_finish_block<T, MODE>(a, ov, lane, X, st);
        }
      }
    }
    __syncthreads();
  }
  if (*s_fail) {
    // a wait gave up: record it, and let the copies still in flight land
    // (bounded) before the CTA's shared memory goes away
    if (threadIdx.x == 0) {
      atomicCAS(a.err, 0, MLSH_ERR_TIMEOUT);
      if (rhs_bytes > 0) ring_wait(bar_rhs, 0, a.polls);
    }
    if (producer && lane == 0) {
      for (int q = max(0, issued - slots); q < issued; ++q)
        ring_wait(bar0 + 8u * (uint32_t)(q & (slots - 1)), (uint32_t)(q >> shift) & 1u,
                  a.polls);
    }
    return;
  }
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) a.out[i] = xs[i];
}

// ---------------------------------------------------------------------------
// Schedules: each block's dependency blocks, counted (FILL = false) or
// written (FILL = true) in ascending order without repeats.  Lower: the
// blocks of the columns < base its rows reference; upper: those >= base+32.
template <bool UPPER, bool FILL>
__global__ void __launch_bounds__(kSweepThreads)
    block_deps_kernel(const int *rp, const int *ci, const int *lo_end, const int *up_beg, int n,
                      unsigned nb, int *cnt, const int *off, int *ids) {
  const int lane = threadIdx.x & 31;
  const unsigned blk = blockIdx.x * kSweepWarps + (threadIdx.x >> 5);
  if (blk >= nb) return;
  const int base = (int)blk * 32;
  const int row = base + lane;
  int j = 0, je = 0;
  if (row < n) {
    if (UPPER) {
      je = rp[row + 1];
      j = up_beg[row];
      while (j < je && ci[j] < base + 32) ++j;
    } else {
      j = rp[row];
      je = lo_end[row];
      int k = j;
      while (k < je && ci[k] < base) ++k;
      je = k;
    }
  }
  // scan-eligible: each row's in-block dependencies are at most the
  // adjacent row
  bool adj = true;
  if (!FILL && row < n) {
    if (UPPER) {
      const int b0 = up_beg[row];
      const int nin = j - b0;  // entries in (row, base + 32)
      adj = nin == 0 || (nin == 1 && ci[b0] == row + 1);
    } else {
      const int le = lo_end[row];
      const int nin = le - je;  // entries in [base, row)
      adj = nin == 0 || (nin == 1 && ci[je] == row - 1);
    }
  }
  const bool scan = __all_sync(kFull, adj);
  constexpr int kNone = 0x7fffffff;
  int cur = j < je ? (ci[j] >> 5) : kNone;
  int count = 0;
  const int o = FILL ? off[blk] : 0;
  while (true) {
    const int m = __reduce_min_sync(kFull, cur);
    if (m == kNone) break;
    if (FILL && lane == 0) ids[o + count] = m;
    ++count;
    if (cur == m) {
      while (j < je && (ci[j] >> 5) == m) ++j;
      cur = j < je ? (ci[j] >> 5) : kNone;
    }
  }
  if (!FILL && lane == 0) cnt[blk] = count | (scan ? (1 << 30) : 0);
}

// ---------------------------------------------------------------------------
// Factorizations: one warp per 32-row block, blocks in the lower sweep's
// level order with per-block flags (the sweeps' schedule and protocol).
// Each lane factors its own row with the sequential algorithm's operations
// in the sequential order: first the eliminations by rows outside the block
// (all lanes at once, after the block's dependency blocks are final), then
// those by rows inside the block as a 32-step chain -- at step s row base+s
// is final and every lane whose row stores (i, base+s) applies it.
template <typename T>
struct FactorArgs {
  const int *rp;
  const int *ci;
  const int *lo_end;
  const int *up_beg;
  T *f;  // A's values on entry, the factor on exit
  int n;
  unsigned nb;
  unsigned long long *ticket;
  unsigned *flags;  // nb block flags, zero on entry (one launch: epoch 1)
  const int *order;
  const int *dep_off;
  const int *dep_ids;
  int *err;
  unsigned long long *pivot;  // first zero pivot (min row), ~0 if none
};

// ILU(0) elimination of row `row` by row k (the stored (row, k) at q):
//   a_ik = a_ik / a_kk;  a_ij -= a_ik * a_kj  for stored j > k with a_kj stored
// (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 10.4);
// row k's upper part and row i's later entries are merged in column order.
template <typename T>
__device__ __forceinline__ void ilu_eliminate(const FactorArgs<T> &a, int row, int q, int k) {
  T *f = a.f;
  const int kd = a.lo_end[k], kb = a.up_beg[k], ke = a.rp[k + 1];
  const T ukk = kb > kd ? __ldcg(f + kd) : T(0);
  const T l = div_rn(__ldcg(f + q), ukk);
  f[q] = l;
  const int re = a.rp[row + 1];
  int pos = kb;
  for (int p = q + 1; p < re; ++p) {
    const int c = a.ci[p];
    while (pos < ke && a.ci[pos] < c) ++pos;
    if (pos < ke && a.ci[pos] == c) f[p] = sub_rn(__ldcg(f + p), mul_rn(l, __ldcg(f + pos)));
  }
}

// IC(0) entry l_ik = (a_ik - sum_{m<k} l_im l_km) / l_kk over the stored m of
// both rows, ascending in m.
template <typename T>
__device__ __forceinline__ void ic_entry(const FactorArgs<T> &a, int row, int q, int k) {
  T *f = a.f;
  T acc = __ldcg(f + q);
  const int kd = a.lo_end[k];
  int pk = a.rp[k];
  for (int p = a.rp[row]; p < q; ++p) {
    const int m = a.ci[p];
    while (pk < kd && a.ci[pk] < m) ++pk;
    if (pk < kd && a.ci[pk] == m) acc = sub_rn(acc, mul_rn(__ldcg(f + p), __ldcg(f + pk)));
  }
  const T lkk = a.up_beg[k] > kd ? __ldcg(f + kd) : T(0);
  f[q] = div_rn(acc, lkk);
}

// IC(0) diagonal l_ii = sqrt(a_ii - sum_{m<i} l_im^2), ascending in m.
template <typename T>
__device__ __forceinline__ void ic_diag(const FactorArgs<T> &a, int row) {
  T *f = a.f;
  const int le = a.lo_end[row];
  const bool has = a.up_beg[row] > le;
  T d = has ? __ldcg(f + le) : T(0);
  for (int p = a.rp[row]; p < le; ++p) {
    const T v = __ldcg(f + p);
    d = sub_rn(d, mul_rn(v, v));
  }
  if (!(d > T(0))) atomicMin(a.pivot, (unsigned long long)row);
  if (has) f[le] = sqrt_rn(d);
}

template <typename T, bool IC>
__global__ void __launch_bounds__(kSweepThreads) factor_kernel(FactorArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const unsigned gw = blockIdx.x * kSweepWarps + (threadIdx.x >> 5);
  if (gw >= a.nb) return;
  unsigned long long v = 0;
  if (lane == 0) v = atomicAdd(a.ticket, 1ull);
  const unsigned long long t = __shfl_sync(kFull, v, 0);
  const unsigned epoch = (unsigned)(t / a.nb) + 1u;
  const unsigned blk = (unsigned)a.order[t % a.nb] & kBlockMask;
  const int base = (int)blk * 32;
  const int row = base + lane;
  const bool valid = row < a.n;
  wait_deps(a.dep_off, a.dep_ids, a.flags, blk, epoch, a.err, lane, kWaitPolls);
  int q = valid ? a.rp[row] : 0;
  const int le = valid ? a.lo_end[row] : 0;
  // rows outside the block, ascending
  for (; q < le; ++q) {
    const int k = a.ci[q];
    if (k >= base) break;
    if constexpr (IC) ic_entry(a, row, q, k);
    else ilu_eliminate(a, row, q, k);
  }
  // rows inside the block: the chain
  for (int st = 0; st < 32; ++st) {
    if constexpr (IC) {
      if (lane == st && valid) ic_diag(a, row);
    }
    __syncwarp();
    if (q < le && a.ci[q] == base + st) {
      if constexpr (IC) ic_entry(a, row, q, base + st);
      else ilu_eliminate(a, row, q, base + st);
      ++q;
    }
  }
  __syncwarp();
  if constexpr (!IC) {
    if (valid) {
      const int d = a.lo_end[row];
      if (!(a.up_beg[row] > d) || __ldcg(a.f + d) == T(0))
        atomicMin(a.pivot, (unsigned long long)row);
    }
  }
  publish_block(a.flags + blk, epoch, lane);
}

int grid_of(long long n, int threads) { return (int)std::max<long long>(1, (n + threads - 1) / threads); }

template <typename T, int MODE, bool BWD>
cudaError_t cta_launch(const SweepArgs<T> &a, const Schedule &sc, size_t xbytes, cudaStream_t s) {
  if (sc.ring > 0) {
    const size_t bytes = ring_smem_bytes<T>(a.n, sc.levels, sc.ring);
    sweep_ring_kernel<T, MODE, BWD><<<1, kCtaThreads, bytes, s>>>(
        a, sc.level_off, sc.levels, static_cast<const unsigned char *>(sc.rec), sc.ring);
  } else {
    sweep_cta_kernel<T, MODE, BWD><<<1, kCtaThreads, xbytes, s>>>(a, sc.level_off, sc.levels);
  }
  return cudaGetLastError();
}

// The single-CTA sweeps opt in to 200 KB of shared memory; set once, outside
// any stream capture (the sweeps are captured into solver graphs).
template <typename T>
cudaError_t configure_cta_t() {
  const int bytes = (int)kCtaSweepBytes;
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_cta_kernel<T, kSorFwd, false>, at, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_cta_kernel<T, kUnitFwd, false>, at, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_cta_kernel<T, kDiagFwd, false>, at, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_cta_kernel<T, kSorBwd, true>, at, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_cta_kernel<T, kDiagBwd, true>, at, bytes);
  const int rb = (int)kRingSweepBytes;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_ring_kernel<T, kSorFwd, false>, at, rb);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_ring_kernel<T, kUnitFwd, false>, at, rb);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_ring_kernel<T, kDiagFwd, false>, at, rb);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_ring_kernel<T, kSorBwd, true>, at, rb);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_ring_kernel<T, kDiagBwd, true>, at, rb);
  return e;
}

int configure_cta() {
  static int done = 0;
  if (done) return MLSH_SUCCESS;
  MLSH_CUDA_TRY(configure_cta_t<double>());
  MLSH_CUDA_TRY(configure_cta_t<float>());
  done = 1;
  return MLSH_SUCCESS;
}

template <typename T>
cudaError_t sweep_launch_t(const Precond &pc, const Sweep &sw, bool backward, const void *rhs,
                           void *out, const int *done, int *err, cudaStream_t s) {
  SweepArgs<T> a;
  a.rp = sw.rp;
  a.ci = sw.ci;
  a.val = static_cast<const T *>(sw.val);
  a.lo_end = sw.lo_end;
  a.up_beg = sw.up_beg;
  a.scale = static_cast<const T *>(sw.scale);
  a.rhs = static_cast<const T *>(rhs);
  a.out = static_cast<T *>(out);
  a.n = pc.n;
  a.nb = pc.nb;
  a.ticket = pc.ticket;
  a.flags = pc.flags;
  a.done = done;
  a.err = err;
  a.order = sw.order;
  a.dep_off = sw.dep_off;
  a.dep_ids = sw.dep_ids;
  a.polls = pc.wait_polls;
  const Schedule &sc = backward ? pc.sbwd : pc.sfwd;
  const size_t xbytes = cta_smem_bytes<T>(pc.n, pc.nb, sc.levels);
  if (xbytes <= kCtaSweepBytes) {
    switch (sw.mode) {
      case kSorFwd: return cta_launch<T, kSorFwd, false>(a, sc, xbytes, s);
      case kUnitFwd: return cta_launch<T, kUnitFwd, false>(a, sc, xbytes, s);
      case kDiagFwd: return cta_launch<T, kDiagFwd, false>(a, sc, xbytes, s);
      case kSorBwd: return cta_launch<T, kSorBwd, true>(a, sc, xbytes, s);
      default: return cta_launch<T, kDiagBwd, true>(a, sc, xbytes, s);
    }
  }
  const int g = grid_of(pc.nb, kSweepWarps);
  switch (sw.mode) {
    case kSorFwd: sweep_kernel<T, kSorFwd, false><<<g, kSweepThreads, 0, s>>>(a); break;
    case kUnitFwd: sweep_kernel<T, kUnitFwd, false><<<g, kSweepThreads, 0, s>>>(a); break;
    case kDiagFwd: sweep_kernel<T, kDiagFwd, false><<<g, kSweepThreads, 0, s>>>(a); break;
    case kSorBwd: sweep_kernel<T, kSorBwd, true><<<g, kSweepThreads, 0, s>>>(a); break;
    default: sweep_kernel<T, kDiagBwd, true><<<g, kSweepThreads, 0, s>>>(a); break;
  }
  return cudaGetLastError();
}

template <typename T>
int factor_run(Handle &h, Precond &pc, const int *rp, const int *ci) {
  cudaStream_t s = h.stream;
  unsigned *rowflag = nullptr;  // block flags of the factorization launch
  unsigned long long *scratch = nullptr;  // [ticket, pivot]
  MLSH_CUDA_TRY(pool_alloc(&rowflag, sizeof(unsigned) * (size_t)std::max(pc.nb, 1u), s));
  MLSH_CUDA_TRY(pool_alloc(&scratch, 2 * sizeof(unsigned long long), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(rowflag, 0, sizeof(unsigned) * (size_t)std::max(pc.nb, 1u), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(scratch + 1, 0xff, sizeof(unsigned long long), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(h.err_flag, 0, sizeof(int), s));
  FactorArgs<T> a;
  a.rp = rp;
  a.ci = ci;
  a.lo_end = pc.lo_end;
  a.up_beg = pc.up_beg;
  a.f = static_cast<T *>(pc.fval);
  a.n = pc.n;
  a.nb = pc.nb;
  a.ticket = scratch;
  a.flags = rowflag;
  a.order = pc.sfwd.order;
  a.dep_off = pc.sfwd.dep_off;
  a.dep_ids = pc.sfwd.dep_ids;
  a.err = h.err_flag;
  a.pivot = scratch + 1;
  const int g = grid_of(pc.nb, kSweepWarps);
  if (pc.kind == MLSH_PRECOND_IC) factor_kernel<T, true><<<g, kSweepThreads, 0, s>>>(a);
  else factor_kernel<T, false><<<g, kSweepThreads, 0, s>>>(a);
  MLSH_CUDA_TRY(cudaGetLastError());
  unsigned long long piv = 0;
  int err = 0;
  MLSH_CUDA_TRY(cudaMemcpyAsync(&piv, scratch + 1, sizeof(piv), cudaMemcpyDeviceToHost, s));
  MLSH_CUDA_TRY(cudaMemcpyAsync(&err, h.err_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  pool_free(rowflag, s);
  pool_free(scratch, s);
  if (err != 0) return err;
  if (pc.pivot < 0 && piv != ~0ull) pc.pivot = (long long)piv;
  return MLSH_SUCCESS;
}

}  // namespace

cudaError_t sweep_launch(const Precond &pc, const Sweep &sw, bool backward, const void *rhs,
                         void *out, const int *done, int *err, cudaStream_t s) {
  if (pc.n == 0) return cudaSuccess;
  if (pc.dtype == MLSH_F64) return sweep_launch_t<double>(pc, sw, backward, rhs, out, done, err, s);
  return sweep_launch_t<float>(pc, sw, backward, rhs, out, done, err, s);
}

cudaError_t precond_apply_launch(const Precond &pc, const void *r, void *z, const int *done,
                                 int *err, cudaStream_t s) {
  cudaError_t e = sweep_launch(pc, pc.fwd, false, r, pc.tmp, done, err, s);
  if (e != cudaSuccess) return e;
  return sweep_launch(pc, pc.bwd, true, pc.tmp, z, done, err, s);
}

void precond_release(Precond &pc) {
  cudaStream_t s = pc.handle ? pc.handle->stream : nullptr;
  void *bufs[] = {pc.lo_end,        pc.up_beg,        pc.fval,          pc.rp_t,
                  pc.ci_t,          pc.val_t,         pc.lo_t,          pc.up_t,
                  pc.scale,         pc.tmp,           pc.ticket,        pc.flags,
                  pc.sfwd.order,    pc.sfwd.dep_off,  pc.sfwd.dep_ids,  pc.sbwd.order,
                  pc.sbwd.dep_off,  pc.sbwd.dep_ids,  pc.sfwd.level_off, pc.sbwd.level_off,
                  pc.sfwd.rec,      pc.sbwd.rec};
  for (void *b : bufs) pool_free(b, s);
  pc.sfwd = Schedule{};
  pc.sbwd = Schedule{};
  pc.lo_end = pc.up_beg = pc.rp_t = pc.ci_t = pc.lo_t = pc.up_t = nullptr;
  pc.fval = pc.val_t = pc.scale = pc.tmp = nullptr;
  pc.ticket = nullptr;
  pc.flags = nullptr;
}

namespace {

// lo_end / up_beg of a pattern; MLSH_ERR_INVALID_CSR if a row is not
// sorted; *missing = first row without a stored diagonal (or ~0).
int split_rows(Handle &h, const int *rp, const int *ci, int n, int *lo_end, int *up_beg,
               unsigned long long *missing) {
  cudaStream_t s = h.stream;
  struct Flags {
    unsigned long long missing;
    int bad;
    int pad;
  };
  Flags *d = nullptr;
  MLSH_CUDA_TRY(pool_alloc(&d, sizeof(Flags), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(d, 0xff, sizeof(unsigned long long), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(&d->bad, 0, 2 * sizeof(int), s));
  split_rows_kernel<<<grid_of(n, 256), 256, 0, s>>>(rp, ci, n, lo_end, up_beg, &d->bad,
                                                    &d->missing);
  MLSH_CUDA_TRY(cudaGetLastError());
  Flags hf;
  MLSH_CUDA_TRY(cudaMemcpyAsync(&hf, d, sizeof(Flags), cudaMemcpyDeviceToHost, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  pool_free(d, s);
  if (hf.bad) return MLSH_ERR_INVALID_CSR;
  *missing = hf.missing;
  return MLSH_SUCCESS;
}

// The level schedule of one sweep direction: dependency blocks per block
// on the device, levels and the level order computed on the host (one pass
// over the block DAG in dependency order).
int build_schedule(Handle &h, const int *rp, const int *ci, const int *lo, const int *up, int n,
                   unsigned nb, bool upper, Schedule &sc) {
  cudaStream_t s = h.stream;
  if (nb == 0) return MLSH_SUCCESS;
  const int g = grid_of(nb, kSweepWarps);
  MLSH_CUDA_TRY(pool_alloc(&sc.dep_off, sizeof(int) * ((size_t)nb + 1), s));
  MLSH_CUDA_TRY(pool_alloc(&sc.order, sizeof(int) * (size_t)nb, s));
  int *cnt = sc.order;  // the counts pass borrows the order array
  if (upper)
    block_deps_kernel<true, false><<<g, kSweepThreads, 0, s>>>(rp, ci, lo, up, n, nb, cnt,
                                                                nullptr, nullptr);
  else
    block_deps_kernel<false, false><<<g, kSweepThreads, 0, s>>>(rp, ci, lo, up, n, nb, cnt,
                                                                 nullptr, nullptr);
  MLSH_CUDA_TRY(cudaGetLastError());
  std::vector<int> hc(nb), off((size_t)nb + 1, 0);
  MLSH_CUDA_TRY(cudaMemcpyAsync(hc.data(), cnt, sizeof(int) * (size_t)nb,
                                cudaMemcpyDeviceToHost, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  long long total = 0;
  std::vector<char> scan(nb);
  for (unsigned b = 0; b < nb; ++b) {
    scan[b] = (hc[b] >> 30) & 1;
    hc[b] &= (1 << 30) - 1;
    off[b] = (int)total;
    total += hc[b];
  }
  off[nb] = (int)total;
  sc.deps = total;
  MLSH_CUDA_TRY(pool_alloc(&sc.dep_ids, sizeof(int) * (size_t)std::max(total, 1ll), s));
  MLSH_CUDA_TRY(cudaMemcpyAsync(sc.dep_off, off.data(), sizeof(int) * ((size_t)nb + 1),
                                cudaMemcpyHostToDevice, s));
  if (upper)
    block_deps_kernel<true, true><<<g, kSweepThreads, 0, s>>>(rp, ci, lo, up, n, nb, nullptr,
                                                               sc.dep_off, sc.dep_ids);
  else
    block_deps_kernel<false, true><<<g, kSweepThreads, 0, s>>>(rp, ci, lo, up, n, nb, nullptr,
                                                                sc.dep_off, sc.dep_ids);
  MLSH_CUDA_TRY(cudaGetLastError());
  std::vector<int> ids((size_t)std::max(total, 1ll));
  MLSH_CUDA_TRY(cudaMemcpyAsync(ids.data(), sc.dep_ids, sizeof(int) * (size_t)total,
                                cudaMemcpyDeviceToHost, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  // level = 1 + the highest level among the dependencies (0 without any)
  std::vector<int> lvl(nb, 0);
  int levels = 0;
  for (unsigned k = 0; k < nb; ++k) {
    const unsigned b = upper ? nb - 1 - k : k;
    int m = -1;
    for (int d = off[b]; d < off[b + 1]; ++d) m = std::max(m, lvl[(size_t)ids[d]]);
    lvl[b] = m + 1;
    levels = std::max(levels, m + 2);
  }
  sc.levels = levels;
  // blocks by level (within a level in sweep direction)
  std::vector<int> start((size_t)levels + 1, 0), order(nb);
  for (unsigned b = 0; b < nb; ++b) ++start[(size_t)lvl[b] + 1];
  sc.width = 0;
  for (int l = 0; l < levels; ++l) sc.width = std::max(sc.width, start[(size_t)l + 1]);
  for (int l = 0; l < levels; ++l) start[(size_t)l + 1] += start[(size_t)l];
  MLSH_CUDA_TRY(pool_alloc(&sc.level_off, sizeof(int) * ((size_t)levels + 1), s));
  MLSH_CUDA_TRY(cudaMemcpyAsync(sc.level_off, start.data(), sizeof(int) * ((size_t)levels + 1),
                                cudaMemcpyHostToDevice, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  for (unsigned k = 0; k < nb; ++k) {
    const unsigned b = upper ? nb - 1 - k : k;
    order[(size_t)start[(size_t)lvl[b]]++] = (int)(b | (scan[b] ? kScanBit : 0u));
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(sc.order, order.data(), sizeof(int) * (size_t)nb,
                                cudaMemcpyHostToDevice, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  return MLSH_SUCCESS;
}

int build_impl(Handle &h, const CsrPlan &p, int kind, double omega, bool solver_scale,
               Precond &pc) {
  cudaStream_t s = h.stream;
  const int n = p.n_rows;
  const size_t esz = (size_t)dtype_size(p.dtype);
  int cst = configure_cta();
  if (cst != MLSH_SUCCESS) return cst;
  pc.handle = &h;
  pc.plan = &p;
  pc.kind = kind;
  pc.dtype = p.dtype;
  pc.n = n;
  pc.nnz = p.nnz;
  pc.nb = (unsigned)((n + 31) / 32);
  const size_t nn = (size_t)std::max(n, 1);
  MLSH_CUDA_TRY(pool_alloc(&pc.lo_end, sizeof(int) * nn, s));
  MLSH_CUDA_TRY(pool_alloc(&pc.up_beg, sizeof(int) * nn, s));
  MLSH_CUDA_TRY(pool_alloc(&pc.tmp, esz * nn, s));
  MLSH_CUDA_TRY(pool_alloc(&pc.ticket, sizeof(unsigned long long), s));
  MLSH_CUDA_TRY(pool_alloc(&pc.flags, sizeof(unsigned) * std::max<size_t>(pc.nb, 1), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(pc.ticket, 0, sizeof(unsigned long long), s));
  MLSH_CUDA_TRY(cudaMemsetAsync(pc.flags, 0, sizeof(unsigned) * std::max<size_t>(pc.nb, 1), s));
  if (n == 0) {
    MLSH_CUDA_TRY(cudaStreamSynchronize(s));
    return MLSH_SUCCESS;
  }
  unsigned long long missing = ~0ull;
  int st = split_rows(h, p.row_ptr, p.col_ind, n, pc.lo_end, pc.up_beg, &missing);
  if (st != MLSH_SUCCESS) return st;
  st = build_schedule(h, p.row_ptr, p.col_ind, pc.lo_end, pc.up_beg, n, pc.nb, false, pc.sfwd);
  if (st != MLSH_SUCCESS) return st;
  if (kind != MLSH_PRECOND_IC && !solver_scale) {
    st = build_schedule(h, p.row_ptr, p.col_ind, pc.lo_end, pc.up_beg, n, pc.nb, true, pc.sbwd);
    if (st != MLSH_SUCCESS) return st;
  }
  if (kind == MLSH_PRECOND_SOR) {
    // M = 1/(omega d) for the preconditioner; 1/((1/omega) d) for the solver
    MLSH_CUDA_TRY(pool_alloc(&pc.scale, esz * nn, s));
    if (p.dtype == MLSH_F64) {
      const double w = solver_scale ? 1.0 / omega : omega;
      sor_scale_kernel<double><<<grid_of(n, 256), 256, 0, s>>>(
          static_cast<const double *>(p.val), pc.lo_end, pc.up_beg, n, w,
          static_cast<double *>(pc.scale));
    } else {
      const float of = (float)omega;
      const float w = solver_scale ? (float)(1.0 / (double)of) : of;
      sor_scale_kernel<float><<<grid_of(n, 256), 256, 0, s>>>(
          static_cast<const float *>(p.val), pc.lo_end, pc.up_beg, n, w,
          static_cast<float *>(pc.scale));
    }
    MLSH_CUDA_TRY(cudaGetLastError());
    pc.fwd = Sweep{p.row_ptr,     p.col_ind,       p.val,          pc.lo_end, pc.up_beg,
                   pc.scale,      kSorFwd,         pc.sfwd.order,  pc.sfwd.dep_off,
                   pc.sfwd.dep_ids};
    pc.bwd = Sweep{p.row_ptr,     p.col_ind,       p.val,          pc.lo_end, pc.up_beg,
                   pc.scale,      kSorBwd,         pc.sbwd.order,  pc.sbwd.dep_off,
                   pc.sbwd.dep_ids};
    MLSH_CUDA_TRY(cudaStreamSynchronize(s));
    return MLSH_SUCCESS;
  }
  if (missing != ~0ull) {
    pc.pivot = (long long)missing;
    pc.structural = 1;
  }
  MLSH_CUDA_TRY(pool_alloc(&pc.fval, esz * (size_t)std::max(p.nnz, 1), s));
  if (p.nnz > 0)
    MLSH_CUDA_TRY(cudaMemcpyAsync(pc.fval, p.val, esz * (size_t)p.nnz,
                                  cudaMemcpyDeviceToDevice, s));
  st = p.dtype == MLSH_F64 ? factor_run<double>(h, pc, p.row_ptr, p.col_ind)
                           : factor_run<float>(h, pc, p.row_ptr, p.col_ind);
  if (st != MLSH_SUCCESS) return st;
  if (kind == MLSH_PRECOND_ILU) {
    pc.fwd = Sweep{p.row_ptr,     p.col_ind,       pc.fval,        pc.lo_end, pc.up_beg,
                   nullptr,       kUnitFwd,        pc.sfwd.order,  pc.sfwd.dep_off,
                   pc.sfwd.dep_ids};
    pc.bwd = Sweep{p.row_ptr,     p.col_ind,       pc.fval,        pc.lo_end, pc.up_beg,
                   nullptr,       kDiagBwd,        pc.sbwd.order,  pc.sbwd.dep_off,
                   pc.sbwd.dep_ids};
    return MLSH_SUCCESS;
  }
  // IC: L^T as the rows of the factor's transpose (its upper triangle)
  MLSH_CUDA_TRY(pool_alloc(&pc.rp_t, sizeof(int) * (nn + 1), s));
  MLSH_CUDA_TRY(pool_alloc(&pc.ci_t, sizeof(int) * (size_t)std::max(p.nnz, 1), s));
  MLSH_CUDA_TRY(pool_alloc(&pc.val_t, esz * (size_t)std::max(p.nnz, 1), s));
  MLSH_CUDA_TRY(pool_alloc(&pc.lo_t, sizeof(int) * nn, s));
  MLSH_CUDA_TRY(pool_alloc(&pc.up_t, sizeof(int) * nn, s));
  st = transpose_build(h, n, n, p.nnz, p.row_ptr, p.col_ind, pc.fval, p.dtype, pc.rp_t,
                       pc.ci_t, pc.val_t, nullptr);
  if (st != MLSH_SUCCESS) return st;
  unsigned long long missing_t = ~0ull;
  st = split_rows(h, pc.rp_t, pc.ci_t, n, pc.lo_t, pc.up_t, &missing_t);
  if (st != MLSH_SUCCESS) return st;
  st = build_schedule(h, pc.rp_t, pc.ci_t, pc.lo_t, pc.up_t, n, pc.nb, true, pc.sbwd);
  if (st != MLSH_SUCCESS) return st;
  pc.fwd = Sweep{p.row_ptr,     p.col_ind,       pc.fval,        pc.lo_end, pc.up_beg,
                 nullptr,       kDiagFwd,        pc.sfwd.order,  pc.sfwd.dep_off,
                 pc.sfwd.dep_ids};
  pc.bwd = Sweep{pc.rp_t,       pc.ci_t,         pc.val_t,       pc.lo_t,   pc.up_t,
                 nullptr,       kDiagBwd,        pc.sbwd.order,  pc.sbwd.dep_off,
                 pc.sbwd.dep_ids};
  return MLSH_SUCCESS;
}

}  // namespace

namespace {

// The ring form of one sweep's single-CTA kernel, where it applies: the
// solution fits in shared memory beside a ring of at least kRingMinSlots
// slots, at least twice the widest level (so a level's and the next level's
// records are all in flight at once).
template <typename T>
int build_records_t(Handle &h, const Precond &pc, const Sweep &sw, Schedule &sc) {
  sc.ring = 0;
  if (sc.order == nullptr || pc.nb == 0 || sc.levels == 0) return MLSH_SUCCESS;
  if (cta_smem_bytes<T>(pc.n, pc.nb, sc.levels) > kCtaSweepBytes) return MLSH_SUCCESS;
  int slots = kRingMaxSlots;
  while (slots >= kRingMinSlots && ring_smem_bytes<T>(pc.n, sc.levels, slots) > kRingSweepBytes)
    slots >>= 1;
  if (slots < kRingMinSlots || slots < 2 * sc.width) return MLSH_SUCCESS;
  cudaStream_t s = h.stream;
  MLSH_CUDA_TRY(pool_alloc(&sc.rec, (size_t)SweepRec<T>::kBytes * pc.nb, s));
  SweepArgs<T> a{};
  a.rp = sw.rp;
  a.ci = sw.ci;
  a.val = static_cast<const T *>(sw.val);
  a.lo_end = sw.lo_end;
  a.up_beg = sw.up_beg;
  a.scale = static_cast<const T *>(sw.scale);
  a.n = pc.n;
  a.nb = pc.nb;
  a.order = sw.order;
  unsigned char *rec = static_cast<unsigned char *>(sc.rec);
  const int g = grid_of(pc.nb, kSweepWarps);
  switch (sw.mode) {
    case kSorFwd: sweep_rec_kernel<T, kSorFwd, false><<<g, kSweepThreads, 0, s>>>(a, rec); break;
    case kUnitFwd: sweep_rec_kernel<T, kUnitFwd, false><<<g, kSweepThreads, 0, s>>>(a, rec); break;
    case kDiagFwd: sweep_rec_kernel<T, kDiagFwd, false><<<g, kSweepThreads, 0, s>>>(a, rec); break;
    case kSorBwd: sweep_rec_kernel<T, kSorBwd, true><<<g, kSweepThreads, 0, s>>>(a, rec); break;
    default: sweep_rec_kernel<T, kDiagBwd, true><<<g, kSweepThreads, 0, s>>>(a, rec); break;
  }
  MLSH_CUDA_TRY(cudaGetLastError());
  sc.ring = slots;
  return MLSH_SUCCESS;
}

int build_records(Handle &h, Precond &pc) {
  int st = MLSH_SUCCESS;
  if (pc.dtype == MLSH_F64) {
    st = build_records_t<double>(h, pc, pc.fwd, pc.sfwd);
    if (st == MLSH_SUCCESS) st = build_records_t<double>(h, pc, pc.bwd, pc.sbwd);
  } else {
    st = build_records_t<float>(h, pc, pc.fwd, pc.sfwd);
    if (st == MLSH_SUCCESS) st = build_records_t<float>(h, pc, pc.bwd, pc.sbwd);
  }
  if (st == MLSH_SUCCESS) MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return st;
}

}  // namespace

int precond_build(Handle &h, const CsrPlan &p, int kind, double omega, bool solver_scale,
                  Precond &out) {
  int st = build_impl(h, p, kind, omega, solver_scale, out);
  if (st == MLSH_SUCCESS) st = build_records(h, out);
  if (st != MLSH_SUCCESS) {
    cudaGetLastError();
    precond_release(out);
  }
  return st;
}

}  // namespace mlsh

using namespace mlsh;

// ===================================================================== C ABI
extern "C" {

int mlsh_precond_create(mlsh_handle hs, mlsh_csr_plan ps, int kind, double omega,
                        mlsh_precond *out) {
  if (!hs || !ps || !out) return MLSH_ERR_INVALID_ARG;
  *out = nullptr;
  if (kind != MLSH_PRECOND_SOR && kind != MLSH_PRECOND_IC && kind != MLSH_PRECOND_ILU)
    return MLSH_ERR_INVALID_ARG;
  const CsrPlan &p = ps->p;
  if (p.n_rows != p.n_cols) return MLSH_ERR_INVALID_ARG;
  if (kind == MLSH_PRECOND_SOR && !(omega == omega)) return MLSH_ERR_INVALID_ARG;
  auto *pc = new (std::nothrow) mlsh_precond_s;
  if (!pc) return MLSH_ERR_OOM;
  const int st = precond_build(hs->h, p, kind, omega, false, pc->p);
  if (st != MLSH_SUCCESS) {
    delete pc;
    return st;
  }
  *out = pc;
  return MLSH_SUCCESS;
}

int mlsh_precond_zero_pivot(mlsh_precond pc, int64_t *row, int *structural) {
  if (!pc || !row) return MLSH_ERR_INVALID_ARG;
  *row = pc->p.pivot;
  if (structural) *structural = pc->p.pivot >= 0 ? pc->p.structural : 0;
  return MLSH_SUCCESS;
}

int mlsh_precond_apply(mlsh_handle hs, mlsh_precond pc, const void *r, void *z) {
  if (!hs || !pc) return MLSH_ERR_INVALID_ARG;
  const Precond &p = pc->p;
  if (p.n == 0) return MLSH_SUCCESS;
  if (!r || !z || r == z) return MLSH_ERR_INVALID_ARG;
  Handle &h = hs->h;
  MLSH_CUDA_TRY(cudaMemsetAsync(h.err_flag, 0, sizeof(int), h.stream));
  MLSH_CUDA_TRY(precond_apply_launch(p, r, z, nullptr, h.err_flag, h.stream));
  int err = 0;
  MLSH_CUDA_TRY(cudaMemcpyAsync(&h.host_scalars[7], h.err_flag, sizeof(int),
                                cudaMemcpyDeviceToHost, h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  std::memcpy(&err, &h.host_scalars[7], sizeof(int));
  return err;
}

int mlsh_precond_factor(mlsh_handle hs, mlsh_precond pc, void *out) {
  if (!hs || !pc || !out) return MLSH_ERR_INVALID_ARG;
  const Precond &p = pc->p;
  const size_t esz = (size_t)dtype_size(p.dtype);
  Handle &h = hs->h;
  if (p.kind == MLSH_PRECOND_SOR) {
    if (p.n > 0)
      MLSH_CUDA_TRY(cudaMemcpyAsync(out, p.scale, esz * (size_t)p.n, cudaMemcpyDeviceToDevice,
                                    h.stream));
  } else if (p.nnz > 0) {
    MLSH_CUDA_TRY(cudaMemcpyAsync(out, p.fval, esz * (size_t)p.nnz, cudaMemcpyDeviceToDevice,
                                  h.stream));
  }
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return MLSH_SUCCESS;
}

int mlsh_precond_sweep_form(mlsh_precond pc, int *lower, int *upper) {
  if (!pc) return MLSH_ERR_INVALID_ARG;
  const Precond &p = pc->p;
  auto form = [&](const Schedule &sc) {
    if (sc.order == nullptr) return -1;
    if (sc.ring > 0) return MLSH_SWEEP_RING;
    const size_t bytes = p.dtype == MLSH_F64 ? cta_smem_bytes<double>(p.n, p.nb, sc.levels)
                                             : cta_smem_bytes<float>(p.n, p.nb, sc.levels);
    return bytes <= kCtaSweepBytes ? MLSH_SWEEP_CTA : MLSH_SWEEP_FLAGS;
  };
  if (lower) *lower = form(p.sfwd);
  if (upper) *upper = form(p.sbwd);
  return MLSH_SUCCESS;
}

int mlsh_precond_info(mlsh_precond pc, int *levels_lower, int *levels_upper, int64_t *blocks) {
  if (!pc) return MLSH_ERR_INVALID_ARG;
  if (levels_lower) *levels_lower = pc->p.sfwd.levels;
  if (levels_upper) *levels_upper = pc->p.sbwd.levels;
  if (blocks) *blocks = pc->p.nb;
  return MLSH_SUCCESS;
}

int mlsh_precond_destroy(mlsh_precond pc) {
  if (!pc) return MLSH_SUCCESS;
  if (pc->p.handle) {
    purge_precond_graphs(*pc->p.handle, &pc->p);
    cudaStreamSynchronize(pc->p.handle->stream);
  }
  precond_release(pc->p);
  delete pc;
  return MLSH_SUCCESS;
}

}  // extern "C"
