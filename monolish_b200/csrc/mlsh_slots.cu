// Offset-slot layout and SpMV for the FP32 copy the mixed-precision solver
// iterates on.
//
// The FP32 copy is data derived from the caller's CRS (values rounded to
// FP32, Jacobi folded in); its layout is this library's choice.  Matrices
// that use at most kMaxSlots distinct column offsets (col - row) in all --
// stencil matrices on structured grids, boundary rows included -- keep the
// offsets once and store each slice of kSlotRows rows as one contiguous
// record (mlsh_internal.cuh: a presence mask byte per row, then the values
// slot by slot), so column indices cost nothing per entry and a row costs
// 4 K + 1 bytes (a 7-point
// row: 25 with the unit diagonal implicit, against 46 in CRS with 16-bit
// columns).  When every diagonal value of the copy is exactly 1 (Jacobi
// folded in: a_ii * (1 / a_ii) rounds to 1 in FP32) the diagonal is not
// stored and x_i is added in its place.
//
// The SpMV streams the records like the CRS kernel streams its tiles: a
// producer warp moves each slice's record into a ring of shared-memory
// stages with one 1-D bulk copy (L2 evict-first, so the gathered x stays in
// L2) completing on an mbarrier, and 8 consumer warps, one thread per row,
// read the row from shared memory, release the stage, gather x (the
// offsets are launch parameters) and write y.  (Staging each slot's x run
// with a bulk copy of its own, nine 1 KB copies per slice, measured slower:
// the copies' issue rate, not HBM, then bounds the kernel.)
//
// A matrix qualifies only if every row is sorted, has no repeated column
// and at most kShortRow entries: then each row is summed by one thread in
// ascending column order with separately rounded products -- exactly what
// the CRS kernel does for such rows -- so y does not depend on the layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <new>
#include <vector>

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

struct SlotTable {
  int offs[kMaxSlots];
};

__global__ void __launch_bounds__(kSlotRows)
    slots_fill(int n, const int *rp, const int *ci, const float *val, SlotTable tab, int K,
               int unit, unsigned char *recs) {
  const int slice = blockIdx.x;
  unsigned char *rec = recs + (size_t)slice * slot_rec_bytes(K);
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
        if (s < K && tab.offs[s] == off) {
          v[s] = val[j];
          m |= 1u << s;
        }
    }
  }
  rec[threadIdx.x] = (unsigned char)m;
  float *vals = reinterpret_cast<float *>(rec + kSlotHeadBytes);
#pragma unroll
  for (int s = 0; s < kMaxSlots; ++s)
    if (s < K) vals[s * kSlotRows + threadIdx.x] = v[s];
}

struct SlotArgs {
  const unsigned char *recs;
  int offs[kMaxSlots];      // the matrix's offsets (the first KS used)
  int slot_win[kMaxSlots];  // window of each slot
  int win_lo[kMaxSlotWin];
  int win_len[kMaxSlotWin];
  int win_off[kMaxSlotWin];
  int n_win;
  int diag_win;
  int lo_min;              // smallest window start (relative to a stage's first row)
  int xo[kMaxSlots];       // unclipped stages: byte offset of slot q's value of row 0
  int xdo;                 // ... of the diagonal's
  int w0o, w1o;            // ... of the dot weights'
  unsigned xal;            // bit q: slot q's offset is 16-byte aligned; bit 8: the diagonal's
  unsigned fullm;          // a thread's rows' mask bytes with every slot present
  int yal;                 // y is 16-byte aligned
  int dpos;  // unit diagonal: its place among the slots (the count of negative offsets)
  int w_off;
  int stage_bytes;
  int stages;
  int unit;
  int n_rows;
  int n_slices;
  int n_groups;
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
  int *err;  // set to MLSH_ERR_TIMEOUT if a wait gives up
};

constexpr int kSlotConsumers = kSlotRows;            // one thread per row of a slice
constexpr int kSlotThreads = kSlotConsumers + 32;   // + the producer warp
constexpr int kGroupRows = kSlotGroup * kSlotRows;
constexpr int kWRunBytes = 4 * kGroupRows + 16;     // a weight run, rounded ends
constexpr int kSlotRowsPerThread = kGroupRows / kSlotConsumers;  // consecutive rows
static_assert(kSlotRowsPerThread == 2 || kSlotRowsPerThread == 4, "vector width");
// after the stages: mbarriers, reduction scratch, flags
constexpr int kSlotTailBytes = 2 * kMaxSlotStages * 8 + 32 * 8 + 16 * 4;
constexpr int kSlotFlagAbort = 0;
constexpr int kSlotFlagLast = 1;
constexpr int kSlotFlagWarpDone = 2;  // 8 slots: stages each consumer warp has read

__device__ __forceinline__ float ld_shared_f32(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}

__device__ __forceinline__ float2 ld_shared_f32x2(uint32_t addr) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}

// N consecutive floats of shared memory at `addr` (aligned to 4 N bytes)
template <int N>
__device__ __forceinline__ void ld_shared_vec(uint32_t addr, float (&o)[N]);
template <>
__device__ __forceinline__ void ld_shared_vec<2>(uint32_t addr, float (&o)[2]) {
  const float2 t = ld_shared_f32x2(addr);
  o[0] = t.x; o[1] = t.y;
}
// two consecutive floats to global memory (aligned to 8 bytes)
__device__ __forceinline__ void st_global_vec(float *p, const float (&o)[2]) {
  *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]);
}

// Elements [a, a + len) of v clipped to [0, n): the first element s0, the
// bytes of the 16-byte-rounded copy (0 if empty) and its source.  The
// rounded range never leaves the 16-byte chunks holding elements s0 and
// e0 - 1, so it stays inside the memory that holds v.
__device__ __forceinline__ uint32_t clip_range(const float *v, long long a, int len, int n,
                                               uintptr_t *src) {
  const long long lo = a < 0 ? 0 : a;
  const long long hi = a + len > n ? n : a + len;
  if (hi <= lo) {
    *src = 0;
    return 0;
  }
  const uintptr_t b = (uintptr_t)(v + lo) & ~(uintptr_t)15;
  const uintptr_t e = ((uintptr_t)(v + hi) + 15) & ~(uintptr_t)15;
  *src = b;
  return (uint32_t)(e - b);
}
// Element index (of v) of the first staged element of the copy of [a, ...).
__device__ __forceinline__ long long staged_base(const float *v, long long a) {
  const long long lo = a < 0 ? 0 : a;
  return lo - (long long)(((uintptr_t)(v + lo) & 15u) >> 2);
}

// A persistent grid walks the stages (kSlotGroup slices each); KS = the
// plan's slot count.  Consumer thread ct handles row ct of each slice of a
// stage, reading mask, values, x and the dot weights from shared memory.
// The fused dots accumulate in a fixed per-thread order and are reduced
// like the vector kernels' sums (fixed order, last CTA finalises).  Every
// wait is bounded: a consumer warp that gives up records MLSH_ERR_TIMEOUT
// and stops; the producer then waits for its copies in flight and exits.
// DP: where the implicit unit diagonal goes among the slots, known at
// compile time (symmetric stencils: KS / 2), or kDpRuntime to read it from
// the launch (a.unit, a.dpos).
constexpr int kDpRuntime = -1;

template <int KS, int DP, int M0, int M1>
__global__ void __launch_bounds__(kSlotThreads, 2) spmv_slots_kernel(const SlotArgs a) {
  constexpr int NR = (M0 != kDotNone ? 1 : 0) + (M1 != kDotNone ? 1 : 0);
  constexpr int NA = NR > 0 ? NR : 1;
  constexpr int NW = (M0 == kDotW ? 1 : 0) + (M1 == kDotW ? 1 : 0);
  extern __shared__ __align__(128) unsigned char smem[];
  pdl_wait();
  pdl_launch_dependents();
  if (a.done != nullptr && *a.done != 0) return;
  const int STG = a.stages;
  const int rec_bytes = slot_rec_bytes(KS);
  unsigned char *tail = smem + STG * a.stage_bytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(tail);
  double *red = reinterpret_cast<double *>(tail + 2 * kMaxSlotStages * 8);
  volatile int *flags =
      reinterpret_cast<volatile int *>(tail + 2 * kMaxSlotStages * 8 + 32 * 8);
  const int tid = threadIdx.x;
  const uint32_t full0 = smem_addr(bars);
  const uint32_t empty0 = smem_addr(bars + kMaxSlotStages);
  if (tid == 0) {
    for (int s = 0; s < STG; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, kSlotConsumers / 32);  // one arrival per consumer warp
    }
    for (int f = 0; f < 16; ++f) flags[f] = 0;
    fence_mbar_init();
  }
  __syncthreads();
  const float *wv0 = (M0 == kDotW) ? a.w0 : a.w1;  // first weight run
  const float *wv1 = a.w1;                          // second (both dots weighted)

  if (tid < 32) {
    // ------------------------------------------------------- producer ---
    // lane 0 copies the stage's records; lane 1 + w window w; then the
    // weight runs
    const int lane = tid;
    const uint64_t policy = l2_evict_first_policy();
    int k = 0;
    bool aborted = false;
    for (int g = blockIdx.x; g < a.n_groups; g += gridDim.x, ++k) {
      const int s = k % STG;
      if (k >= STG) {
        int ok = 1;
        if (lane == 0) {
          const uint32_t par = (uint32_t)((k / STG - 1) & 1);
          const uint64_t t0 = global_timer_ns();
          ok = 0;
          for (uint32_t it = 1;; ++it) {
            if (mbar_try_wait_sleep(empty0 + 8 * s, par, 1000u)) { ok = 1; break; }
            if ((it & 7u) == 0 && flags[kSlotFlagAbort]) break;
            if ((it & 63u) == 0 && global_timer_ns() - t0 > kWaitLimitNs) {
              atomicExch(a.err, MLSH_ERR_TIMEOUT);
              break;
            }
          }
        }
        if (__shfl_sync(0xffffffffu, ok, 0) == 0) { aborted = true; break; }
      }
      const int sl0 = g * kSlotGroup;
      const long long R0 = (long long)sl0 * kSlotRows;
      unsigned char *st = smem + s * a.stage_bytes;
      uint32_t bytes = 0, dst = 0;
      uintptr_t src = 0;
      const int j = lane - 1;
      if (lane == 0) {
        const int ns = min(kSlotGroup, a.n_slices - sl0);
        bytes = (uint32_t)(ns * rec_bytes);
        src = (uintptr_t)(a.recs + (size_t)sl0 * rec_bytes);
        dst = smem_addr(st);
      } else if (j < a.n_win) {
        bytes = clip_range(a.x, R0 + a.win_lo[j], a.win_len[j], a.n_rows, &src);
        dst = smem_addr(st + a.win_off[j]);
      } else if (j == a.n_win && NW >= 1) {
        bytes = clip_range(wv0, R0, kGroupRows, a.n_rows, &src);
        dst = smem_addr(st + a.w_off);
      } else if (j == a.n_win + 1 && NW >= 2) {
        bytes = clip_range(wv1, R0, kGroupRows, a.n_rows, &src);
        dst = smem_addr(st + a.w_off + kWRunBytes);
      }
      uint32_t total = bytes;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      const uint32_t bar = full0 + 8 * s;
      if (lane == 0) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, total);
      }
      __syncwarp();
      if (lane == 0)  // the records: read once, evict first (x stays in L2)
        bulk_g2s_hint(dst, (const void *)src, bytes, bar, policy);
      else if (bytes)
        bulk_g2s(dst, (const void *)src, bytes, bar);
    }
    if (lane != 0) return;
    const int issued = k;
    // Tail: the consumers release every issued stage; if they gave up, wait
    // for the copies themselves so that none is in flight at exit.
    for (int kk = issued - STG < 0 ? 0 : issued - STG; kk < issued && !aborted; ++kk) {
      const int s = kk % STG;
      const uint32_t par = (uint32_t)((kk / STG) & 1);
      const uint64_t t0 = global_timer_ns();
      for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(empty0 + 8 * s, par)) break;
        if (((it & 63u) == 0 && flags[kSlotFlagAbort]) ||
            ((it & 1023u) == 0 && global_timer_ns() - t0 > kWaitLimitNs)) {
          aborted = true;
          break;
        }
      }
    }
    if (aborted) {
      atomicExch(a.err, MLSH_ERR_TIMEOUT);
      int consumed = issued;
      for (int w = 0; w < kSlotConsumers / 32; ++w)
        consumed = min(consumed, (int)flags[kSlotFlagWarpDone + w]);
      for (int kk = consumed; kk < issued; ++kk)
        mbar_wait_bounded(full0 + 8 * (kk % STG), (uint32_t)((kk / STG) & 1), kWaitLimitNs);
    }
    return;
  }

  // ---------------------------------------------------------- consumers ---
  const int ct = tid - 32;
  const int lane = ct & 31, warp = ct >> 5;
  double acc[NA];
#pragma unroll
  for (int q = 0; q < NA; ++q) acc[q] = 0.0;
  const bool plain = a.alpha == 1.0 && a.beta == 0.0;
  const bool unit = DP >= 0 || a.unit != 0;
  const int dpos = DP >= 0 ? DP : (a.unit ? a.dpos : kMaxSlots + 1);
  const uint32_t smem0 = smem_addr(smem);
  // thread ct takes rows RPT ct .. RPT ct + RPT - 1 of each stage: slice
  // RPT ct / kSlotRows of the stage, rows sr .. sr + RPT - 1 of that slice
  constexpr int RPT = kSlotRowsPerThread;
  const int lr0 = RPT * ct;
  const int gs = lr0 / kSlotRows;
  const int sr = lr0 % kSlotRows;
  const uint32_t lr4 = 4u * (uint32_t)lr0;
  int k = 0;
  for (int g = blockIdx.x; g < a.n_groups; g += gridDim.x, ++k) {
    const int s = k % STG;
    int ok = 1;
    if (lane == 0) {
      ok = flags[kSlotFlagAbort] == 0 &&
           mbar_wait_sleep_bounded(full0 + 8 * s, (uint32_t)((k / STG) & 1), kWaitLimitNs);
      if (!ok && flags[kSlotFlagAbort] == 0) {
        flags[kSlotFlagAbort] = 1;
        atomicExch(a.err, MLSH_ERR_TIMEOUT);
      }
    }
    if (__shfl_sync(0xffffffffu, ok, 0) == 0) break;
    const unsigned char *st = smem + s * a.stage_bytes;
    const int sl0 = g * kSlotGroup;
    const long long R0 = (long long)sl0 * kSlotRows;
    // per slot: the shared address of the value for local row 0 of this
    // stage.  Stages start on kGroupRows boundaries, so a window's 16-byte
    // rounding is the same in every stage whose window is not clipped at
    // row 0: there the launch's precomputed offsets (and their 16-byte
    // alignment flags) hold; the first stages recompute.
    const uint32_t stg = smem0 + s * a.stage_bytes;
    uint32_t xa[KS > 0 ? KS : 1];
    uint32_t xda = stg + a.xdo;
    unsigned xal = a.xal;
    if (R0 + a.lo_min >= 0) {
#pragma unroll
      for (int q = 0; q < KS; ++q) xa[q] = stg + a.xo[q];
    } else {
      xal = 0;
#pragma unroll
      for (int q = 0; q < KS; ++q)
        xa[q] = stg + a.win_off[a.slot_win[q]] + 4 * a.offs[q] -
                4 * (int)(staged_base(a.x, R0 + a.win_lo[a.slot_win[q]]) - R0);
      if (a.diag_win >= 0)
        xda = stg + a.win_off[a.diag_win] -
              4 * (int)(staged_base(a.x, R0 + a.win_lo[a.diag_win]) - R0);
    }
    const int ns = min(kSlotGroup, a.n_slices - sl0);
    const long long left = a.n_rows - R0 - lr0;
    const int nl = left < RPT ? (int)left : RPT;  // live rows of this thread
    if (gs < ns && nl > 0) {
      const unsigned char *rec = st + gs * rec_bytes;
      const uint32_t m4 = RPT == 4 ? *reinterpret_cast<const uint32_t *>(rec + sr)
                                   : *reinterpret_cast<const uint16_t *>(rec + sr);
      const uint32_t vals = smem_addr(rec + kSlotHeadBytes) + 4 * sr;
      float v[KS > 0 ? KS : 1][RPT], xx[KS > 0 ? KS : 1][RPT], xd[RPT], sum[RPT];
#pragma unroll
      for (int q = 0; q < KS; ++q) ld_shared_vec<RPT>(vals + 4 * q * kSlotRows, v[q]);
      const bool full = m4 == a.fullm;
      // a thread's RPT consecutive values of a window: one vector load when
      // aligned
      auto ld4 = [&](uint32_t ad, bool al, float (&o)[RPT]) {
        if (al) {
          ld_shared_vec<RPT>(ad, o);
        } else {
#pragma unroll
          for (int j = 0; j < RPT; ++j) o[j] = ld_shared_f32(ad + 4 * j);
        }
      };
      if (full) {
#pragma unroll
        for (int q = 0; q < KS; ++q) {
          ld4(xa[q] + lr4, (xal >> q) & 1u, xx[q]);
        }
      } else {
#pragma unroll
        for (int q = 0; q < KS; ++q)
#pragma unroll
          for (int j = 0; j < RPT; ++j)
            xx[q][j] = ((m4 >> (8 * j + q)) & 1u) ? ld_shared_f32(xa[q] + lr4 + 4 * j) : 0.0f;
      }
      if (unit) {
        if (nl == RPT && (xal & (1u << kMaxSlots))) {
          ld_shared_vec<RPT>(xda + lr4, xd);
        } else {
#pragma unroll
          for (int j = 0; j < RPT; ++j) xd[j] = j < nl ? ld_shared_f32(xda + lr4 + 4 * j) : 0.0f;
        }
      }
      // per row: ascending columns, products rounded separately (the CRS
      // row loop); the implicit diagonal after the dpos negative offsets
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        float sj = 0.0f;
#pragma unroll
        for (int q = 0; q < KS; ++q) {
          if (q == dpos) sj = __fadd_rn(sj, xd[j]);
          if (full || ((m4 >> (8 * j + q)) & 1u)) sj = __fadd_rn(sj, __fmul_rn(v[q][j], xx[q][j]));
        }
        if (unit && dpos >= KS) sj = __fadd_rn(sj, xd[j]);
        sum[j] = sj;
      }
      const long long r0 = R0 + lr0;
      float out[RPT];
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        out[j] = sum[j];  // alpha = 1, beta = 0: (float)(1.0 * (double)sum) == sum
        if (!plain && j < nl) {
          const double ds = (double)sum[j];
          out[j] = (a.beta == 0.0) ? (float)(a.alpha * ds)
                                   : (float)(a.alpha * ds + a.beta * (double)a.y_in[r0 + j]);
        }
      }
      if (nl == RPT && a.yal) {
        st_global_vec(a.y_out + r0, out);
      } else {
#pragma unroll
        for (int j = 0; j < RPT; ++j)
          if (j < nl) a.y_out[r0 + j] = out[j];
      }
      float wa[RPT] = {}, wbv[RPT] = {};
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        if constexpr (NW >= 1) wa[j] = j < nl ? ld_shared_f32(stg + a.w0o + lr4 + 4 * j) : 0.0f;
        if constexpr (NW >= 2) wbv[j] = j < nl ? ld_shared_f32(stg + a.w1o + lr4 + 4 * j) : 0.0f;
      }
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        if (j < nl) {
          if constexpr (M0 == kDotW) acc[0] += (double)wa[j] * (double)out[j];
          if constexpr (M0 == kDotSelf) acc[0] += (double)out[j] * (double)out[j];
          if constexpr (M1 == kDotW)
            acc[1] += (double)(M0 == kDotW ? wbv[j] : wa[j]) * (double)out[j];
          if constexpr (M1 == kDotSelf) acc[1] += (double)out[j] * (double)out[j];
        }
      }
    }
    // the warp is done with the stage
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(empty0 + 8 * s);
      flags[kSlotFlagWarpDone + warp] = k + 1;
    }
  }
  if constexpr (NR > 0) {
    group_sum<NA>(acc, red, ct, kSlotConsumers, 1);
    int *sflag = const_cast<int *>(flags + kSlotFlagLast);
    if (publish_partials<NA>(acc, a.partials, a.counter, sflag, ct, kSlotConsumers, 1)) {
      double tot[NA];
      reduce_partials<NA>(tot, a.partials, (int)gridDim.x, nullptr, 0, NA, a.counter, red, ct,
                          kSlotConsumers, 1);
      if (ct == 0) {
#pragma unroll
        for (int q = 0; q < NR; ++q) a.dot_out[q] = tot[q];
      }
    }
  }
}

// Largest dynamic shared memory a slot launch may ask for, and what two
// CTAs on one SM may use together (228 KB per SM, 1 KB reserved per CTA).
constexpr int kSlotSmemMax = 220 * 1024;
constexpr int kSlotSmemPerSm = 226 * 1024;

// Per instantiation, once (outside any stream capture: slots_build calls
// slots_prepare): the shared-memory opt-in.
template <int KS, int DP, int M0, int M1>
struct SlotLaunch {
  static bool ready;
  static cudaError_t prepare() {
    if (ready) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(spmv_slots_kernel<KS, DP, M0, M1>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               kSlotSmemMax);
    if (e == cudaSuccess) ready = true;
    return e;
  }
  static int per_sm(int smem) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, spmv_slots_kernel<KS, DP, M0, M1>,
                                                      kSlotThreads, smem) != cudaSuccess) {
      cudaGetLastError();
      b = 0;
    }
    return b;
  }
  static cudaError_t launch(const SlotArgs &a, int grid, int smem, cudaStream_t stream) {
    return launch_dependent(spmv_slots_kernel<KS, DP, M0, M1>, grid, kSlotThreads, smem, stream,
                            a);
  }
};
template <int KS, int DP, int M0, int M1>
bool SlotLaunch<KS, DP, M0, M1>::ready = false;

template <int KS, int DP>
cudaError_t prepare_modes(int smem, int *min_per_sm) {
  cudaError_t e = SlotLaunch<KS, DP, kDotNone, kDotNone>::prepare();
  if (e == cudaSuccess) e = SlotLaunch<KS, DP, kDotW, kDotNone>::prepare();
  if (e == cudaSuccess) e = SlotLaunch<KS, DP, kDotW, kDotSelf>::prepare();
  if (e == cudaSuccess) e = SlotLaunch<KS, DP, kDotSelf, kDotNone>::prepare();
  if (e != cudaSuccess) return e;
  int b = SlotLaunch<KS, DP, kDotNone, kDotNone>::per_sm(smem);
  b = std::min(b, SlotLaunch<KS, DP, kDotW, kDotNone>::per_sm(smem));
  b = std::min(b, SlotLaunch<KS, DP, kDotW, kDotSelf>::per_sm(smem));
  b = std::min(b, SlotLaunch<KS, DP, kDotSelf, kDotNone>::per_sm(smem));
  *min_per_sm = std::min(*min_per_sm, b);
  return cudaSuccess;
}

template <int KS>
cudaError_t prepare_ks(int smem, int *min_per_sm) {
  *min_per_sm = 1 << 20;
  cudaError_t e = prepare_modes<KS, kDpRuntime>(smem, min_per_sm);
  if constexpr (KS == 4 || KS == 6 || KS == 8)
    if (e == cudaSuccess) e = prepare_modes<KS, KS / 2>(smem, min_per_sm);
  return e;
}

cudaError_t slots_prepare(int K, int smem, int *per_sm) {
  switch (K) {
    case 0: return prepare_ks<0>(smem, per_sm);
    case 1: return prepare_ks<1>(smem, per_sm);
    case 2: return prepare_ks<2>(smem, per_sm);
    case 3: return prepare_ks<3>(smem, per_sm);
    case 4: return prepare_ks<4>(smem, per_sm);
    case 5: return prepare_ks<5>(smem, per_sm);
    case 6: return prepare_ks<6>(smem, per_sm);
    case 7: return prepare_ks<7>(smem, per_sm);
    default: return prepare_ks<8>(smem, per_sm);
  }
}

// The stage plan of a layout with offsets offs[0..K) (+ the diagonal): x
// windows (offsets closer than kSlotMergeGap share one), their places in a
// stage, and the weight runs after them.
void plan_stages(SlotFormat &f) {
  std::vector<std::pair<int, int>> need;  // (offset, slot or -1 for the diagonal)
  for (int q = 0; q < f.K; ++q) need.push_back({f.offs[q], q});
  if (f.unit) need.push_back({0, -1});
  std::sort(need.begin(), need.end());
  f.n_win = 0;
  f.diag_win = -1;
  int bytes = kSlotGroup * slot_rec_bytes(f.K);
  int lo = 0, hi = 0;
  auto close = [&]() {
    const int w = f.n_win - 1;
    f.win_lo[w] = lo;
    f.win_len[w] = hi - lo + kGroupRows;
    f.win_off[w] = bytes;
    // the copy of L elements rounded out to 16-byte boundaries at both ends
    bytes += ((4 * f.win_len[w] + 15) & ~15) + 32;
  };
  for (size_t i = 0; i < need.size(); ++i) {
    const int o = need[i].first;
    if (f.n_win == 0 || (long long)o - hi > kSlotMergeGap) {
      if (f.n_win > 0) close();
      ++f.n_win;
      lo = hi = o;
    } else {
      hi = o;
    }
    if (need[i].second >= 0) f.slot_win[need[i].second] = f.n_win - 1;
    else f.diag_win = f.n_win - 1;
  }
  if (f.n_win > 0) close();
  f.w_off = bytes;
  bytes += 2 * kWRunBytes;
  f.stage_bytes = bytes;
}

}  // namespace

void slots_release(CsrPlan &p) {
  if (!p.slots) return;
  cudaStream_t s = p.handle ? p.handle->stream : nullptr;
  pool_free(p.slots->recs, s);
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
  cudaError_t e = cudaStreamSynchronize(s);
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
  // the offsets of all slices together (a slice's are a subset of these)
  std::vector<int> all((size_t)n_slices * kMaxSlots);
  e = cudaMemcpyAsync(all.data(), offs, sizeof(int) * all.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  pool_free(offs, s);
  if (e != cudaSuccess) {
    set_last_error("slot layout offsets", e);
    return MLSH_ERR_CUDA;
  }
  std::vector<int> uni;
  for (int o : all)
    if (o != kSlotUnused && !(unit && o == 0)) uni.push_back(o);
  std::sort(uni.begin(), uni.end());
  uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
  if ((int)uni.size() > kMaxSlots) return MLSH_SUCCESS;  // not this layout
  const int K = (int)uni.size();
  SlotTable tab;
  for (int q = 0; q < kMaxSlots; ++q) tab.offs[q] = q < K ? uni[q] : 0;
  SlotFormat *f = new (std::nothrow) SlotFormat();
  if (!f) return MLSH_ERR_OOM;
  for (int q = 0; q < kMaxSlots; ++q) f->offs[q] = tab.offs[q];
  f->K = K;
  f->unit = unit;
  f->n_slices = n_slices;
  plan_stages(*f);
  // two CTAs per SM with as many stages each (up to kMaxSlotStages) as fit
  // (twice the consumer warps to hide shared-memory latency), else as many
  // stages as fit one CTA
  {
    const int two = std::min(kMaxSlotStages,
                             (kSlotSmemPerSm / 2 - kSlotTailBytes) / f->stage_bytes);
    f->stages = two >= 2 ? two
                         : std::min(kMaxSlotStages,
                                    (kSlotSmemMax - kSlotTailBytes) / f->stage_bytes);
  }
  int per_sm = 0;
  if (f->stages >= 2) {
    e = slots_prepare(K, f->stages * f->stage_bytes + kSlotTailBytes, &per_sm);
    if (e != cudaSuccess) {
      delete f;
      set_last_error("slot SpMV set-up", e);
      return MLSH_ERR_CUDA;
    }
  }
  if (f->stages < 2 || per_sm < 1) {  // windows too wide: the CRS kernel stays
    delete f;
    return MLSH_SUCCESS;
  }
  f->grid_per_sm = per_sm;
  if (pool_alloc(&f->recs, (size_t)f->bytes(), s) != cudaSuccess) {
    cudaGetLastError();
    delete f;
    return MLSH_SUCCESS;  // no room: the CRS kernel stays
  }
  slots_fill<<<n_slices, kSlotRows, 0, s>>>(n, p.row_ptr, p.col_ind, val, tab, K, unit,
                                            f->recs);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    pool_free(f->recs, s);
    delete f;
    set_last_error("slot layout fill", e);
    return MLSH_ERR_CUDA;
  }
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
  a.recs = f.recs;
  for (int q = 0; q < kMaxSlots; ++q) {
    a.offs[q] = f.offs[q];
    a.slot_win[q] = f.slot_win[q];
  }
  for (int w = 0; w < kMaxSlotWin; ++w) {
    a.win_lo[w] = f.win_lo[w];
    a.win_len[w] = f.win_len[w];
    a.win_off[w] = f.win_off[w];
  }
  a.n_win = f.n_win;
  a.diag_win = f.diag_win;
  // Offsets of unclipped stages: a window of stage R0 starts at element
  // R0 + lo rounded down to 16 bytes, and R0 is a multiple of kGroupRows, so
  // the rounding depends only on lo and the vector's own address.
  auto head = [](const float *v, long long e) {
    return (int)((((uintptr_t)v + 4 * (uintptr_t)e) & 15u) >> 2);
  };
  a.lo_min = 0;
  for (int w = 0; w < f.n_win; ++w) a.lo_min = std::min(a.lo_min, f.win_lo[w]);
  for (int q = 0; q < kMaxSlots; ++q) {
    const int w = f.slot_win[q];
    a.xo[q] = q < f.K ? f.win_off[w] + 4 * f.offs[q] - 4 * (f.win_lo[w] - head(x, f.win_lo[w]))
                      : 0;
  }
  a.xdo = f.diag_win >= 0
              ? f.win_off[f.diag_win] - 4 * (f.win_lo[f.diag_win] - head(x, f.win_lo[f.diag_win]))
              : 0;
  {
    const float *wv0 = (M0 == kDotW) ? w0 : w1;
    a.w0o = f.w_off + 4 * (wv0 ? head(wv0, 0) : 0);
    a.w1o = f.w_off + kWRunBytes + 4 * (w1 ? head(w1, 0) : 0);
  }
  a.dpos = f.unit ? (int)(std::lower_bound(f.offs, f.offs + f.K, 0) - f.offs) : kMaxSlots + 1;
  a.xal = 0;
  for (int q = 0; q < f.K; ++q)
    if ((a.xo[q] & 15) == 0) a.xal |= 1u << q;
  if (f.diag_win >= 0 && (a.xdo & 15) == 0) a.xal |= 1u << kMaxSlots;
  const unsigned mk = f.K >= 8 ? 0xffu : ((1u << f.K) - 1u);
  a.fullm = 0;
  for (int j = 0; j < kSlotRowsPerThread; ++j) a.fullm |= mk << (8 * j);
  a.yal = ((uintptr_t)y_out % (4 * kSlotRowsPerThread)) == 0 ? 1 : 0;
  a.w_off = f.w_off;
  a.stage_bytes = f.stage_bytes;
  a.stages = f.stages;
  a.unit = f.unit;
  a.n_rows = p.n_rows;
  a.n_slices = f.n_slices;
  a.n_groups = (f.n_slices + kSlotGroup - 1) / kSlotGroup;
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
  a.err = h.err_flag;
  const int smem = f.stages * f.stage_bytes + kSlotTailBytes;
  const int grid = std::max(1, std::min({a.n_groups, f.grid_per_sm * h.num_sms,
                                         kMaxPartialBlocks}));
  const bool sym = f.unit && a.dpos == f.K / 2 && (f.K % 2) == 0;
  if (sym && f.K == 4) return SlotLaunch<4, 2, M0, M1>::launch(a, grid, smem, stream);
  if (sym && f.K == 6) return SlotLaunch<6, 3, M0, M1>::launch(a, grid, smem, stream);
  if (sym && f.K == 8) return SlotLaunch<8, 4, M0, M1>::launch(a, grid, smem, stream);
  switch (f.K) {
    case 0: return SlotLaunch<0, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 1: return SlotLaunch<1, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 2: return SlotLaunch<2, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 3: return SlotLaunch<3, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 4: return SlotLaunch<4, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 5: return SlotLaunch<5, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 6: return SlotLaunch<6, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    case 7: return SlotLaunch<7, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
    default: return SlotLaunch<8, kDpRuntime, M0, M1>::launch(a, grid, smem, stream);
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
