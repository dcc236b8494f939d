// Offset-slot layout and SpMV for the FP32 copy the mixed-precision solver
// iterates on.
//
// The FP32 copy is data derived from the caller's CRS (values rounded to
// FP32, Jacobi folded in); its layout is this library's choice.  Matrices
// whose rows, in slices of kSlotRows consecutive rows, use at most
// kMaxSlots distinct column offsets (col - row) -- stencil matrices on
// structured grids, boundary rows included -- are stored as:
//   offs[slice][k]      the slice's offsets, ascending (k < K)
//   vals[slice][k][r]   value of row r's entry at offset offs[k] (0 if absent)
//   mask[slice][r]      bit k set when row r has an entry at offs[k]
// so the column indices cost nothing per entry, every slot of a slice is one
// coalesced 1 KB run of values, and a row costs 4 K + 1 bytes (a 7-point
// row: 25 with the unit diagonal implicit, against 46 in CRS with 16-bit
// columns).  When every diagonal value of the copy is exactly 1 (Jacobi
// folded in: a_ii * (1 / a_ii) rounds to 1 in FP32) the diagonal is not
// stored and x_i is added in its place.
//
// A matrix qualifies only if every row is sorted, has no repeated column
// and at most kShortRow entries: then each row is summed by one thread in
// ascending column order with separately rounded products -- exactly what
// the CRS kernel does for such rows -- so y does not depend on the layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <new>

#include "mlsh_core.cuh"

namespace mlsh {

namespace {

constexpr int kSlotUnused = INT_MIN;

// flags[0]: most slots in a slice; [1]: the same without offset 0;
// [2]: a row disqualifies the layout; [3]: some row's diagonal is not 1.
__global__ void __launch_bounds__(kSlotRows)
    slots_scan(int n, const int *rp, const int *ci, const float *val, int *offs, int *flags) {
  __shared__ int tab[kMaxSlots];
  const int slice = blockIdx.x;
  const int r = slice * kSlotRows + (int)threadIdx.x;
  if (threadIdx.x < kMaxSlots) tab[threadIdx.x] = kSlotUnused;
  __syncthreads();
  int bad = 0, nonunit = 0;
  if (r < n) {
    const int b = rp[r], e = rp[r + 1];
    if (e - b > kShortRow) bad = 1;
    bool diag = false;
    int prev = -1;
    for (int j = b; j < e && !bad; ++j) {
      const int c = ci[j];
      if (c <= prev) {  // unsorted or repeated column
        bad = 1;
        break;
      }
      prev = c;
      const int off = c - r;
      if (off == 0) {
        diag = true;
        if (val[j] != 1.0f) nonunit = 1;
      }
      int s = 0;
      for (; s < kMaxSlots; ++s) {  // lock-free insert into the slice's set
        const int old = atomicCAS(&tab[s], kSlotUnused, off);
        if (old == kSlotUnused || old == off) break;
      }
      if (s == kMaxSlots) bad = 1;
    }
    if (!diag) nonunit = 1;
  }
  if (bad) atomicOr(flags + 2, 1);
  if (nonunit) atomicOr(flags + 3, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int t[kMaxSlots];
    int k = 0;
    for (int s = 0; s < kMaxSlots; ++s)
      if (tab[s] != kSlotUnused) t[k++] = tab[s];
    for (int i = 1; i < k; ++i) {  // insertion sort, ascending
      const int v = t[i];
      int j = i - 1;
      while (j >= 0 && t[j] > v) {
        t[j + 1] = t[j];
        --j;
      }
      t[j + 1] = v;
    }
    int has0 = 0;
    for (int s = 0; s < kMaxSlots; ++s) {
      offs[slice * kMaxSlots + s] = s < k ? t[s] : kSlotUnused;
      if (s < k && t[s] == 0) has0 = 1;
    }
    atomicMax(flags + 0, k);
    atomicMax(flags + 1, k - has0);
  }
}

__global__ void __launch_bounds__(kSlotRows)
    slots_fill(int n, const int *rp, const int *ci, const float *val, int *offs, int K,
               int unit, float *vals, uint8_t *mask) {
  __shared__ int tab[kMaxSlots];
  const int slice = blockIdx.x;
  if (threadIdx.x == 0) {
    int k = 0;
    for (int s = 0; s < kMaxSlots; ++s) {
      const int o = offs[slice * kMaxSlots + s];
      if (o == kSlotUnused || (unit && o == 0)) continue;
      tab[k++] = o;
    }
    for (int s = k; s < kMaxSlots; ++s) tab[s] = kSlotUnused;
  }
  __syncthreads();
  if (threadIdx.x < kMaxSlots) offs[slice * kMaxSlots + threadIdx.x] = tab[threadIdx.x];
  const int r = slice * kSlotRows + (int)threadIdx.x;
  float v[kMaxSlots];
#pragma unroll
  for (int s = 0; s < kMaxSlots; ++s) v[s] = 0.0f;
  unsigned m = 0;
  if (r < n) {
    for (int j = rp[r]; j < rp[r + 1]; ++j) {
      const int off = ci[j] - r;
      if (unit && off == 0) continue;
#pragma unroll
      for (int s = 0; s < kMaxSlots; ++s)
        if (tab[s] == off) {
          v[s] = val[j];
          m |= 1u << s;
        }
    }
  }
#pragma unroll
  for (int s = 0; s < kMaxSlots; ++s)
    if (s < K) vals[((size_t)slice * K + s) * kSlotRows + threadIdx.x] = v[s];
  mask[(size_t)slice * kSlotRows + threadIdx.x] = (uint8_t)m;
}

struct SlotArgs {
  const float *vals;
  const uint8_t *mask;
  const int *offs;
  int K;
  int unit;
  int n_rows;
  int n_slices;
  const float *x;
  float *y_out;
  const float *y_in;  // read only when beta != 0
  double alpha, beta;
  const float *w0;
  const float *w1;
  double *partials;
  unsigned *counter;
  double *dot_out;
  const int *done;
};

// One thread per row; a persistent grid walks the slices.  The next
// slice's mask, offsets and values are loaded while the current slice's x
// gathers are in flight, so HBM always has a slice's stream outstanding
// (without that the kernel waits on each slice's loads, then on its
// gathers).  KS = the plan's slot count.  The fused dots accumulate in a
// fixed per-thread order and are reduced like the vector kernels' sums
// (fixed order, last CTA finalises).
template <int KS>
struct SlotRow {
  unsigned m;
  int off[KS > 0 ? KS : 1];
  float v[KS > 0 ? KS : 1];
};

template <int KS>
__device__ __forceinline__ void slot_load(const SlotArgs &a, int sl, SlotRow<KS> &s) {
  const bool in = sl < a.n_slices;
  s.m = in ? (unsigned)__ldcs(a.mask + (size_t)sl * kSlotRows + threadIdx.x) : 0u;
#pragma unroll
  for (int k = 0; k < KS; ++k) {
    s.off[k] = in ? __ldg(a.offs + sl * kMaxSlots + k) : 0;
    s.v[k] = in ? __ldcs(a.vals + ((size_t)sl * KS + k) * kSlotRows + threadIdx.x) : 0.0f;
  }
}

template <int KS, int M0, int M1>
__global__ void __launch_bounds__(kSlotRows, 4) spmv_slots_kernel(const SlotArgs a) {
  constexpr int NR = (M0 != kDotNone ? 1 : 0) + (M1 != kDotNone ? 1 : 0);
  constexpr int NA = NR > 0 ? NR : 1;
  __shared__ double red[kSlotRows / 32 * NA];
  __shared__ int last_flag;
  pdl_wait();
  pdl_launch_dependents();
  if (a.done != nullptr && *a.done != 0) return;
  double acc[NA];
#pragma unroll
  for (int q = 0; q < NA; ++q) acc[q] = 0.0;
  SlotRow<KS> nxt;
  slot_load<KS>(a, blockIdx.x, nxt);
  for (int sl = blockIdx.x; sl < a.n_slices; sl += gridDim.x) {
    const SlotRow<KS> cur = nxt;
    const int r = sl * kSlotRows + (int)threadIdx.x;
    const bool live = r < a.n_rows;
    float xx[KS > 0 ? KS : 1];
#pragma unroll
    for (int k = 0; k < KS; ++k)
      xx[k] = ((cur.m >> k) & 1u) ? __ldg(a.x + r + cur.off[k]) : 0.0f;
    const float xd = (a.unit && live) ? __ldg(a.x + r) : 0.0f;
    slot_load<KS>(a, sl + (int)gridDim.x, nxt);
    // ascending columns, products rounded separately: the CRS row loop
    float sum = 0.0f;
    bool placed = a.unit == 0;
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      if (!placed && cur.off[k] > 0) {
        sum = __fadd_rn(sum, xd);
        placed = true;
      }
      if ((cur.m >> k) & 1u) sum = __fadd_rn(sum, __fmul_rn(cur.v[k], xx[k]));
    }
    if (!placed) sum = __fadd_rn(sum, xd);
    if (live) {
      const double ds = (double)sum;
      const float out = (a.beta == 0.0) ? (float)(a.alpha * ds)
                                        : (float)(a.alpha * ds + a.beta * (double)a.y_in[r]);
      a.y_out[r] = out;
      if constexpr (M0 == kDotW) acc[0] += (double)a.w0[r] * (double)out;
      if constexpr (M0 == kDotSelf) acc[0] += (double)out * (double)out;
      if constexpr (M1 == kDotW) acc[1] += (double)a.w1[r] * (double)out;
      if constexpr (M1 == kDotSelf) acc[1] += (double)out * (double)out;
    }
  }
  if constexpr (NR > 0) {
    group_sum<NA>(acc, red, threadIdx.x, kSlotRows, 0);
    if (publish_partials<NA>(acc, a.partials, a.counter, &last_flag, threadIdx.x, kSlotRows,
                             0)) {
      double tot[NA];
      reduce_partials<NA>(tot, a.partials, (int)gridDim.x, nullptr, 0, NA, a.counter, red,
                          threadIdx.x, kSlotRows, 0);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NR; ++q) a.dot_out[q] = tot[q];
      }
    }
  }
}

template <int KS, int M0, int M1>
cudaError_t launch_slots_ks(const SlotArgs &a, int num_sms, cudaStream_t stream) {
  static int per_sm = 0;
  constexpr auto k = spmv_slots_kernel<KS, M0, M1>;
  if (per_sm == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, kSlotRows, 0) != cudaSuccess ||
        b < 1) {
      cudaGetLastError();
      b = 1;
    }
    per_sm = b;
  }
  int g = std::min(a.n_slices, per_sm * num_sms);
  g = std::max(std::min(g, kMaxPartialBlocks), 1);
  return launch_dependent(k, g, kSlotRows, 0, stream, a);
}

}  // namespace

void slots_release(CsrPlan &p) {
  if (!p.slots) return;
  cudaStream_t s = p.handle ? p.handle->stream : nullptr;
  pool_free(p.slots->vals, s);
  pool_free(p.slots->mask, s);
  pool_free(p.slots->offs, s);
  delete p.slots;
  p.slots = nullptr;
}

int slots_build(CsrPlan &p, cudaStream_t s) {
  slots_release(p);
  if (p.dtype != MLSH_F32 || p.n_rows <= 0 || p.n_rows != p.n_cols) return MLSH_SUCCESS;
  const int n = p.n_rows;
  const int n_slices = (n + kSlotRows - 1) / kSlotRows;
  int *offs = nullptr, *flags = nullptr;
  if (pool_alloc(&offs, sizeof(int) * (size_t)n_slices * kMaxSlots, s) != cudaSuccess ||
      pool_alloc(&flags, sizeof(int) * 4, s) != cudaSuccess) {
    cudaGetLastError();
    pool_free(offs, s);
    return MLSH_SUCCESS;  // no room: the CRS kernel stays
  }
  MLSH_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int) * 4, s));
  const float *val = static_cast<const float *>(p.val);
  slots_scan<<<n_slices, kSlotRows, 0, s>>>(n, p.row_ptr, p.col_ind, val, offs, flags);
  int hf[4] = {0, 0, 0, 0};
  cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  pool_free(flags, s);
  if (e != cudaSuccess) {
    pool_free(offs, s);
    set_last_error("slot layout scan", e);
    return MLSH_ERR_CUDA;
  }
  if (hf[2] != 0) {  // not this layout
    pool_free(offs, s);
    return MLSH_SUCCESS;
  }
  const int unit = hf[3] == 0 ? 1 : 0;
  const int K = unit ? hf[1] : hf[0];
  SlotFormat *f = new (std::nothrow) SlotFormat();
  if (!f) {
    pool_free(offs, s);
    return MLSH_ERR_OOM;
  }
  f->offs = offs;
  f->K = K;
  f->unit = unit;
  f->n_slices = n_slices;
  if (pool_alloc(&f->vals, sizeof(float) * (size_t)n_slices * std::max(K, 1) * kSlotRows, s) !=
          cudaSuccess ||
      pool_alloc(&f->mask, (size_t)n_slices * kSlotRows, s) != cudaSuccess) {
    cudaGetLastError();
    p.slots = f;
    slots_release(p);
    return MLSH_SUCCESS;
  }
  slots_fill<<<n_slices, kSlotRows, 0, s>>>(n, p.row_ptr, p.col_ind, val, offs, K, unit,
                                            f->vals, f->mask);
  MLSH_CUDA_TRY(cudaGetLastError());
  p.slots = f;
  return MLSH_SUCCESS;
}

template <int M0, int M1>
cudaError_t launch_spmv_slots(const CsrPlan &p, const Handle &h, double alpha, const float *x,
                              double beta, const float *y_in, float *y_out, const float *w0,
                              const float *w1, double *dot_out, const int *done,
                              cudaStream_t stream) {
  const SlotFormat &f = *p.slots;
  SlotArgs a;
  a.vals = f.vals;
  a.mask = f.mask;
  a.offs = f.offs;
  a.K = f.K;
  a.unit = f.unit;
  a.n_rows = p.n_rows;
  a.n_slices = f.n_slices;
  a.x = x;
  a.y_out = y_out;
  a.y_in = y_in;
  a.alpha = alpha;
  a.beta = beta;
  a.w0 = w0;
  a.w1 = w1;
  a.partials = h.partials;
  a.counter = h.counters;
  a.dot_out = dot_out;
  a.done = done;
  switch (f.K) {
    case 0: return launch_slots_ks<0, M0, M1>(a, h.num_sms, stream);
    case 1: return launch_slots_ks<1, M0, M1>(a, h.num_sms, stream);
    case 2: return launch_slots_ks<2, M0, M1>(a, h.num_sms, stream);
    case 3: return launch_slots_ks<3, M0, M1>(a, h.num_sms, stream);
    case 4: return launch_slots_ks<4, M0, M1>(a, h.num_sms, stream);
    case 5: return launch_slots_ks<5, M0, M1>(a, h.num_sms, stream);
    case 6: return launch_slots_ks<6, M0, M1>(a, h.num_sms, stream);
    case 7: return launch_slots_ks<7, M0, M1>(a, h.num_sms, stream);
    default: return launch_slots_ks<8, M0, M1>(a, h.num_sms, stream);
  }
}

#define MLSH_INST_SLOTS(A, B)                                                              \
  template cudaError_t launch_spmv_slots<A, B>(const CsrPlan &, const Handle &, double,  \
                                               const float *, double, const float *,      \
                                               float *, const float *, const float *,     \
                                               double *, const int *, cudaStream_t);
MLSH_INST_SLOTS(kDotNone, kDotNone)
MLSH_INST_SLOTS(kDotW, kDotNone)
MLSH_INST_SLOTS(kDotW, kDotSelf)
MLSH_INST_SLOTS(kDotSelf, kDotNone)
#undef MLSH_INST_SLOTS

}  // namespace mlsh

using namespace mlsh;

extern "C" int mlsh_csr_plan_set_layout(mlsh_csr_plan ps, int layout, int *applied) {
  if (!ps || (layout != MLSH_LAYOUT_CRS && layout != MLSH_LAYOUT_SLOTS))
    return MLSH_ERR_INVALID_ARG;
  CsrPlan &p = ps->p;
  cudaStream_t s = p.handle ? p.handle->stream : nullptr;
  if (layout == MLSH_LAYOUT_CRS) {
    if (p.slots) {
      MLSH_CUDA_TRY(cudaStreamSynchronize(s));  // no launch still reads it
      slots_release(p);
    }
  } else if (!p.slots) {
    if (p.dtype != MLSH_F32) return MLSH_ERR_INVALID_ARG;
    const int st = slots_build(p, s);
    if (st != MLSH_SUCCESS) return st;
    MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (applied) *applied = (layout == MLSH_LAYOUT_SLOTS) == (p.slots != nullptr) ? 1 : 0;
  return MLSH_SUCCESS;
}
