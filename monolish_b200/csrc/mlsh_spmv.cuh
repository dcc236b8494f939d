// CRS SpMV for sm_100a: y_out = alpha*A*x + beta*y_in, optionally fused
// with up to two dot products of the result (w0.y / y.y) reduced to device
// scalars, so solvers get (p, Ap) etc. without another pass over HBM.
//
// Reference behaviour replaced: blas::matvec on matrix::CRS<T>
// (src/blas/matrix/matvec/crs_matvec.hpp:8-114; OSS row loop :101-108).
//
// Design (HBM-bound; no tensor cores -- SpMV is not a dense contraction):
//  * Rows are cut on the host into tiles of <= kTileRows rows and
//    <= kTileNnz nonzeros.  Rows longer than kTileNnz become chunk tiles.
//  * A persistent grid (a few CTAs per SM) walks the tiles round-robin, so
//    every CTA's work and summation order are fixed by the sizes.
//  * Warp specialisation: warp 0 is the producer.  Lane 0 streams each
//    tile's contiguous val[] and col_ind[] ranges into a STAGES-deep ring
//    of shared-memory stages with 1-D bulk (TMA) copies that complete on an
//    mbarrier; the other lanes fill the <16-byte ragged ends with plain
//    loads.  HBM sees only long, aligned, fully used bursts, and the copies
//    carry an L2 evict-first policy so the once-read matrix does not push
//    the gathered x out of L2.
//  * 8 consumer warps.  Each thread first issues the row_ptr loads of its
//    row of the tile (independent of the stage, so they overlap the wait),
//    then:
//      pass A  val[j]*x[col[j]] in place over the tile's nonzeros
//              (nonzero-parallel: the x gathers are balanced and
//              independent; x goes through the read-only path);
//      pass B  one thread sums each row of up to kShortRow entries in row
//              order (the reference's loop order, so those rows are
//              bit-identical to it);
//      pass C  longer rows are cut into kSegW-entry segments spread over
//              all warps (an 8-lane tree per segment, four segments per
//              warp instruction), then each row adds its segment sums in
//              order -- balanced and deterministic;
//      pass D  y written coalesced, fused dots accumulated in a fixed
//              per-thread order.
//  * Chunk tiles reduce their products CTA-wide into a per-chunk partial;
//    the last chunk to arrive (atomic counter per long row) sums the
//    partials in chunk order and writes the row.
//  * Every wait on an mbarrier is bounded; on timeout the CTA records
//    MLSH_ERR_TIMEOUT, drains its in-flight copies and exits.
//  * Variants (pipeline depth x CTAs per SM) trade shared memory against
//    L1 capacity for the x gathers and against occupancy; the plan keeps
//    the one its autotuner measured fastest.
#pragma once
#include "mlsh_internal.cuh"
#include "mlsh_ptx.cuh"
#include "mlsh_reduce.cuh"

namespace mlsh {

// Dot modes for the fused reductions.
constexpr int kDotNone = 0;
constexpr int kDotW = 1;     // sum w[i] * y[i]
constexpr int kDotSelf = 2;  // sum y[i] * y[i]

// Rows longer than kShortRow are summed in segments of kSegW entries.
constexpr int kSegW = 8;
// Upper bound of segments in one tile: each such row has > kSegW entries,
// so ceil(len/kSegW) < 2*len/kSegW.
constexpr int kMaxSegs = 2 * kTileNnz / kSegW;
static_assert(kShortRow >= kSegW, "segments must not be longer than short rows");

template <typename VT, typename XT>
struct SpmvArgs {
  const int *row_ptr;
  const int *col;
  // 16-bit column format: col16[j] = col[j] - tile_base[tile of j]
  const uint16_t *col16;
  const int *tile_base;
  const VT *val;
  const Tile *tiles;
  int n_tiles;
  int n_long;
  const LongRow *longs;
  double *chunk_part;
  unsigned *long_cnt;
  double *long_dot;  // 2 per long row
  const XT *x;
  XT *y_out;
  const XT *y_in;  // read only when beta != 0
  double alpha;
  double beta;
  const XT *w0;
  const XT *w1;
  double *partials;
  unsigned *counter;
  double *dot_out;  // NR results
  const int *done;  // optional: skip the launch when *done != 0
  int *err;         // set to MLSH_ERR_TIMEOUT if a wait gives up
};

template <typename VT, int STAGES, int CSZ = 4>
struct SpmvSmem {
  // a tile's range rounded out to 16-byte boundaries: at most 32 extra bytes
  static constexpr int kValBytes = ((kTileNnz * (int)sizeof(VT) + 32) + 15) & ~15;
  static constexpr int kColBytes = ((kTileNnz * CSZ + 32) + 15) & ~15;
  static constexpr int kStageBytes = kValBytes + kColBytes;
  static constexpr int kYsOff = STAGES * kStageBytes;
  static constexpr int kSegSumOff = kYsOff + kTileRows * (int)sizeof(VT) + 16;
  static constexpr int kSegIdxOff = kSegSumOff + kMaxSegs * (int)sizeof(VT) + 16;
  static constexpr int kBarOff = (kSegIdxOff + 2 * kMaxSegs * 2 + 64 + 15) & ~15;
  static constexpr int kRedOff = kBarOff + 2 * STAGES * 8;
  static constexpr int kFlagOff = kRedOff + 32 * 8;
  static constexpr int kBytes = kFlagOff + 16 * 4;
};

// flags[] in shared memory
constexpr int kFlagProdAbort = 0;
constexpr int kFlagConsAbort = 1;
constexpr int kFlagConsumed = 2;
constexpr int kFlagLast = 3;
constexpr int kFlagWarpSeg = 4;  // 8 per-warp segment counts (4..11)

template <typename T>
__device__ __forceinline__ T spmv_mul_rn(T a, T b) {
  if constexpr (sizeof(T) == 8) return __dmul_rn(a, b);
  else return __fmul_rn(a, b);
}
template <typename T>
__device__ __forceinline__ T spmv_add_rn(T a, T b) {
  if constexpr (sizeof(T) == 8) return __dadd_rn(a, b);
  else return __fadd_rn(a, b);
}

template <typename T>
__device__ __forceinline__ int head_elems(const T *base, int idx) {
  return (int)(((uintptr_t)(base + idx) & 15u) / sizeof(T));
}

// Named barrier over the consumer threads that also ORs a predicate.
__device__ __forceinline__ bool consumers_sync_or(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "n"(kConsumers)
      : "memory");
  return r != 0;
}

// Producer side: the bulk copy of a tile's [nb, ne) range of `arr` covers
// the range rounded out to 16-byte boundaries (what a bulk copy needs), so
// element nb lands at element offset head_elems(arr, nb) of the stage.  The
// rounded range never leaves the 16-byte chunks holding elements nb and
// ne-1, so it stays inside memory that holds the array.
template <typename E>
__device__ __forceinline__ uint32_t rounded_range(const E *arr, int nb, int ne, uintptr_t *src) {
  if (ne <= nb) {
    *src = 0;
    return 0;
  }
  const uintptr_t lo = (uintptr_t)(arr + nb) & ~(uintptr_t)15;
  const uintptr_t hi = ((uintptr_t)(arr + ne) + 15) & ~(uintptr_t)15;
  *src = lo;
  return (uint32_t)(hi - lo);
}

// C16: columns stored as 16-bit offsets from a per-tile base (2 bytes per
// nonzero instead of 4) -- the plan picks it when every tile's columns span
// fewer than 65,536 values.
template <typename VT, typename XT, int M0, int M1, int STAGES, int MINB, bool C16 = false>
__global__ void __launch_bounds__(kSpmvThreads, MINB)
    spmv_tiles_kernel(const SpmvArgs<VT, XT> a) {
  constexpr int NR = (M0 != kDotNone ? 1 : 0) + (M1 != kDotNone ? 1 : 0);
  using L = SpmvSmem<VT, STAGES, C16 ? 2 : 4>;
  extern __shared__ __align__(128) unsigned char smem[];
  if (a.done != nullptr && *a.done != 0) return;

  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::kBarOff);
  double *red = reinterpret_cast<double *>(smem + L::kRedOff);
  volatile int *flags = reinterpret_cast<volatile int *>(smem + L::kFlagOff);
  VT *ys = reinterpret_cast<VT *>(smem + L::kYsOff);
  VT *segsum = reinterpret_cast<VT *>(smem + L::kSegSumOff);
  short *seg_lo = reinterpret_cast<short *>(smem + L::kSegIdxOff);
  short *seg_hi = seg_lo + kMaxSegs;
  const int tid = threadIdx.x;
  const uint32_t full0 = smem_addr(bars);
  const uint32_t empty0 = smem_addr(bars + STAGES);

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, kConsumers / 32);  // one arrival per consumer warp
    }
    for (int f = 0; f < 16; ++f) flags[f] = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (tid < 32) {
    // ------------------------------------------------------- producer ---
    const int lane = tid;
    const uint64_t stream_policy = l2_evict_first_policy();
    int k = 0;
    bool aborted = false;
    Tile tl_next = {0, 0, 0, 0, 0, {0, 0, 0}};
    if ((int)blockIdx.x < a.n_tiles) tl_next = a.tiles[blockIdx.x];
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++k) {
      const int s = k % STAGES;
      const Tile tl = tl_next;
      // the next tile's record is in flight while this one is issued
      if (t + (int)gridDim.x < a.n_tiles) tl_next = a.tiles[t + gridDim.x];
      if (k >= STAGES) {
        int ok = 1;
        if (lane == 0) {
          const uint32_t par = (uint32_t)((k / STAGES - 1) & 1);
          const uint64_t t0 = global_timer_ns();
          ok = 0;
          while (true) {
            if (mbar_try_wait(empty0 + 8 * s, par)) { ok = 1; break; }
            if (flags[kFlagConsAbort]) break;
            if (global_timer_ns() - t0 > kWaitLimitNs) {
              atomicExch(a.err, MLSH_ERR_TIMEOUT);
              break;
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) { aborted = true; break; }
      }
      if (lane == 0) {
        unsigned char *st = smem + s * L::kStageBytes;
        const uint32_t bar = full0 + 8 * s;
        uintptr_t vsrc, csrc;
        const uint32_t vb = rounded_range<VT>(a.val, tl.nnz_begin, tl.nnz_end, &vsrc);
        uint32_t cb;
        if constexpr (C16)
          cb = rounded_range<uint16_t>(a.col16, tl.nnz_begin, tl.nnz_end, &csrc);
        else
          cb = rounded_range<int>(a.col, tl.nnz_begin, tl.nnz_end, &csrc);
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, vb + cb);
        if (vb) bulk_g2s_hint(smem_addr(st), (const void *)vsrc, vb, bar, stream_policy);
        if (cb)
          bulk_g2s_hint(smem_addr(st + L::kValBytes), (const void *)csrc, cb, bar, stream_policy);
      }
      __syncwarp();
    }
    const int issued = k;
    // Tail: wait until the consumers have released every issued stage (so
    // no copy is in flight when the CTA exits).  If they aborted, wait for
    // the copies themselves instead.
    if (lane == 0) {
      for (int kk = issued - STAGES < 0 ? 0 : issued - STAGES; kk < issued; ++kk) {
        const int s = kk % STAGES;
        const uint32_t par = (uint32_t)((kk / STAGES) & 1);
        const uint64_t t0 = global_timer_ns();
        bool ok = false;
        while (true) {
          if (mbar_try_wait(empty0 + 8 * s, par)) { ok = true; break; }
          if (flags[kFlagConsAbort]) break;
          if (global_timer_ns() - t0 > kWaitLimitNs) break;
        }
        if (!ok) { aborted = true; break; }
      }
      if (aborted) {
        atomicExch(a.err, MLSH_ERR_TIMEOUT);
        const int consumed = flags[kFlagConsumed];
        for (int kk = consumed; kk < issued; ++kk) {
          const int s = kk % STAGES;
          mbar_wait_bounded(full0 + 8 * s, (uint32_t)((kk / STAGES) & 1), kWaitLimitNs);
        }
      }
    }
    return;
  }

  // ---------------------------------------------------------- consumers ---
  const int ct = tid - 32;  // consumer thread id 0..255
  const int lane = ct & 31, warp = ct >> 5;
  double acc[NR > 0 ? NR : 1];
#pragma unroll
  for (int q = 0; q < (NR > 0 ? NR : 1); ++q) acc[q] = 0.0;
  const double alpha = a.alpha, beta = a.beta;
  constexpr int kPer = kTileNnz / kConsumers;  // 7 products per thread

  // Per-tile values each thread needs besides the staged val/col: the tile
  // record, its row bounds, the 16-bit column base and the fused dot's
  // w0 entry.  They are fetched one tile ahead (the record two steps
  // ahead), so their latency hides behind the current tile's gathers.
  Tile tl_c = {0, 0, 0, 0};
  int g0c = 0, g1c = 0, cbc = 0;
  XT w0c = XT(0);
  {
    const int t0 = blockIdx.x;
    if (t0 < a.n_tiles) {
      tl_c = a.tiles[t0];
      const int nr = tl_c.row_end >= 0 ? tl_c.row_end - tl_c.row_begin : 0;
      if (ct < nr) {
        g0c = __ldg(a.row_ptr + tl_c.row_begin + ct);
        g1c = __ldg(a.row_ptr + tl_c.row_begin + ct + 1);
        if constexpr (M0 == kDotW) w0c = a.w0[tl_c.row_begin + ct];
      }
      if constexpr (C16) cbc = __ldg(a.tile_base + t0);
    }
  }

  int k = 0;
  for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++k) {
    const int s = k % STAGES;
    const Tile tl = tl_c;
    const bool normal = tl.row_end >= 0;
    const int rb = tl.row_begin;
    const int nrows = normal ? tl.row_end - tl.row_begin : 0;
    const int g0 = g0c, g1 = g1c;
    const int col_base = cbc;
    const XT w0v = w0c;
    const int tn = t + (int)gridDim.x;
    Tile tl_n = {0, -1, 0, 0};
    if (tn < a.n_tiles) tl_n = a.tiles[tn];
    if (ct == 0) {
      if (!mbar_wait_bounded(full0 + 8 * s, (uint32_t)((k / STAGES) & 1), kWaitLimitNs)) {
        flags[kFlagConsAbort] = 1;
        atomicExch(a.err, MLSH_ERR_TIMEOUT);
      }
    }
    named_sync(1, kConsumers);
    if (flags[kFlagConsAbort]) break;

    const int nb = tl.nnz_begin, ne = tl.nnz_end, nt = ne - nb;
    unsigned char *st = smem + s * L::kStageBytes;
    VT *v = reinterpret_cast<VT *>(st) + head_elems(a.val, nb);

    if (normal && tl.short_only) {
      // ---------------------------------------------- direct: short rows
      // Every row has <= kShortRow entries: each thread gathers and sums
      // its own row in row order with separately rounded products (the
      // reference's loop, as passes A+B compute it), with no exchange
      // through shared memory and no barrier before the stage is released.
      VT sum = VT(0);
      if (ct < nrows) {
        const int s0 = g0 - nb, len = g1 - g0;
        XT xx[kShortRow];
        if constexpr (C16) {
          const uint16_t *c = reinterpret_cast<const uint16_t *>(st + L::kValBytes) +
                              head_elems(a.col16, nb);
#pragma unroll
          for (int u = 0; u < kShortRow; ++u)
            if (u < len) xx[u] = __ldg(a.x + col_base + (int)c[s0 + u]);
        } else {
          const int *c = reinterpret_cast<const int *>(st + L::kValBytes) + head_elems(a.col, nb);
#pragma unroll
          for (int u = 0; u < kShortRow; ++u)
            if (u < len) xx[u] = __ldg(a.x + c[s0 + u]);
        }
#pragma unroll
        for (int u = 0; u < kShortRow; ++u)
          if (u < len) sum = spmv_add_rn(sum, spmv_mul_rn(v[s0 + u], (VT)xx[u]));
      }
      // this warp is done with the stage
      __syncwarp();
      if (lane == 0) mbar_arrive(empty0 + 8 * s);
      if (ct == 0) flags[kFlagConsumed] = k + 1;
      if (ct < nrows) {
        const int r = rb + ct;
        const double dsum = (double)sum;
        const XT out = (beta == 0.0) ? (XT)(alpha * dsum)
                                     : (XT)(alpha * dsum + beta * (double)a.y_in[r]);
        a.y_out[r] = out;
        if constexpr (M0 == kDotW) acc[0] += (double)w0v * (double)out;
        if constexpr (M0 == kDotSelf) acc[0] += (double)out * (double)out;
        if constexpr (M1 == kDotW) acc[1] += (double)a.w1[r] * (double)out;
        if constexpr (M1 == kDotSelf) acc[1] += (double)out * (double)out;
      }
      // prefetch the next tile's per-thread values
      g0c = g1c = cbc = 0;
      w0c = XT(0);
      if (tn < a.n_tiles) {
        const int nr = tl_n.row_end >= 0 ? tl_n.row_end - tl_n.row_begin : 0;
        if (ct < nr) {
          g0c = __ldg(a.row_ptr + tl_n.row_begin + ct);
          g1c = __ldg(a.row_ptr + tl_n.row_begin + ct + 1);
          if constexpr (M0 == kDotW) w0c = a.w0[tl_n.row_begin + ct];
        }
        if constexpr (C16) cbc = __ldg(a.tile_base + tn);
      }
      tl_c = tl_n;
      continue;
    }

    // pass A: products in place
    {
      int cc[kPer];
      XT xx[kPer];
      if constexpr (C16) {
        const uint16_t *c = reinterpret_cast<const uint16_t *>(st + L::kValBytes) +
                            head_elems(a.col16, nb);
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
          const int j = ct + u * kConsumers;
          cc[u] = (j < nt) ? col_base + (int)c[j] : 0;
        }
      } else {
        const int *c = reinterpret_cast<const int *>(st + L::kValBytes) + head_elems(a.col, nb);
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
          const int j = ct + u * kConsumers;
          cc[u] = (j < nt) ? c[j] : 0;
        }
      }
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int j = ct + u * kConsumers;
        xx[u] = (j < nt) ? __ldg(a.x + cc[u]) : XT(0);
      }
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int j = ct + u * kConsumers;
        if (j < nt) v[j] = v[j] * (VT)xx[u];
      }
    }
    named_sync(1, kConsumers);
    // prefetch the next tile's per-thread values
    g0c = g1c = cbc = 0;
    w0c = XT(0);
    if (tn < a.n_tiles) {
      const int nr = tl_n.row_end >= 0 ? tl_n.row_end - tl_n.row_begin : 0;
      if (ct < nr) {
        g0c = __ldg(a.row_ptr + tl_n.row_begin + ct);
        g1c = __ldg(a.row_ptr + tl_n.row_begin + ct + 1);
        if constexpr (M0 == kDotW) w0c = a.w0[tl_n.row_begin + ct];
      }
      if constexpr (C16) cbc = __ldg(a.tile_base + tn);
    }
    tl_c = tl_n;

    if (normal) {
      // ------------------------------------------------ pass B: short rows
      const int s0 = g0 - nb, s1 = g1 - nb, len = s1 - s0;
      const bool med = ct < nrows && len > kShortRow;
      if (ct < nrows && !med) {
        VT sum = VT(0);
        for (int j = s0; j < s1; ++j) sum += v[j];
        ys[ct] = sum;
      }
      // ------------------------------------ pass C: kSegW-entry segments
      if (consumers_sync_or(med)) {
        // exclusive scan of segment counts over the tile's rows
        const int nseg = med ? (len + kSegW - 1) / kSegW : 0;
        int inc = nseg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += y;
        }
        if (lane == 31) flags[kFlagWarpSeg + warp] = inc;
        named_sync(1, kConsumers);
        int base = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kConsumers / 32; ++w) {
          const int cw = flags[kFlagWarpSeg + w];
          if (w < warp) base += cw;
          total += cw;
        }
        const int first = base + inc - nseg;
        for (int q = 0; q < nseg; ++q) {
          seg_lo[first + q] = (short)(s0 + kSegW * q);
          seg_hi[first + q] = (short)min(s0 + kSegW * (q + 1), s1);
        }
        named_sync(1, kConsumers);
        // four segments per warp step: lanes 8g..8g+7 take segment g
        constexpr int kSegPerWarp = 32 / kSegW;
        const int sub = lane / kSegW, sl = lane % kSegW;
        for (int sg0 = warp * kSegPerWarp; sg0 < total; sg0 += kConsumers / kSegW) {
          const int sg = sg0 + sub;
          VT part = VT(0);
          if (sg < total) {
            const int j = seg_lo[sg] + sl;
            if (j < seg_hi[sg]) part = v[j];
          }
#pragma unroll
          for (int o = kSegW / 2; o > 0; o >>= 1)
            part += __shfl_xor_sync(0xffffffffu, part, o, kSegW);
          if (sl == 0 && sg < total) segsum[sg] = part;
        }
        named_sync(1, kConsumers);
        if (med) {
          VT sum = VT(0);
          for (int q = 0; q < nseg; ++q) sum += segsum[first + q];
          ys[ct] = sum;
        }
      }
      // all reads of the stage are done (the last barrier above)
      if (lane == 0) mbar_arrive(empty0 + 8 * s);
      if (ct == 0) flags[kFlagConsumed] = k + 1;
      // ----------------------------------------------------- pass D: y
      if (ct < nrows) {
        const int r = rb + ct;
        const double sum = (double)ys[ct];
        const XT out = (beta == 0.0) ? (XT)(alpha * sum)
                                     : (XT)(alpha * sum + beta * (double)a.y_in[r]);
        a.y_out[r] = out;
        if constexpr (M0 == kDotW) acc[0] += (double)w0v * (double)out;
        if constexpr (M0 == kDotSelf) acc[0] += (double)out * (double)out;
        if constexpr (M1 == kDotW) acc[1] += (double)a.w1[r] * (double)out;
        if constexpr (M1 == kDotSelf) acc[1] += (double)out * (double)out;
      }
    } else {
      // --------------------------------------------- chunk of a long row ---
      VT part = VT(0);
      for (int j = ct; j < nt; j += kConsumers) part += v[j];
      part = warp_sum(part);
      if (lane == 0) red[warp] = (double)part;
      named_sync(1, kConsumers);
      if (lane == 0) mbar_arrive(empty0 + 8 * s);
      if (ct == 0) {
        flags[kFlagConsumed] = k + 1;
        double tot = 0.0;
        for (int w = 0; w < kConsumers / 32; ++w) tot += red[w];
        const int li = -tl.row_end - 1;
        const LongRow lr = a.longs[li];
        const int row = lr.row;
        const int slot = lr.first_slot + (nb - __ldg(a.row_ptr + row)) / kTileNnz;
        a.chunk_part[slot] = tot;
        __threadfence();
        const unsigned prev = atomicAdd(a.long_cnt + li, 1u);
        if (prev == (unsigned)(lr.n_chunks - 1)) {
          __threadfence();
          double sum = 0.0;
          for (int q = 0; q < lr.n_chunks; ++q) sum += __ldcg(a.chunk_part + lr.first_slot + q);
          const double ysum = (double)(VT)sum;
          const XT out = (beta == 0.0) ? (XT)(alpha * ysum)
                                       : (XT)(alpha * ysum + beta * (double)a.y_in[row]);
          a.y_out[row] = out;
          double d0 = 0.0, d1 = 0.0;
          if constexpr (M0 == kDotW) d0 = (double)a.w0[row] * (double)out;
          if constexpr (M0 == kDotSelf) d0 = (double)out * (double)out;
          if constexpr (M1 == kDotW) d1 = (double)a.w1[row] * (double)out;
          if constexpr (M1 == kDotSelf) d1 = (double)out * (double)out;
          if constexpr (NR > 0) {
            a.long_dot[2 * li] = d0;
            a.long_dot[2 * li + 1] = d1;
          }
          a.long_cnt[li] = 0u;
        }
      }
    }
  }

  if constexpr (NR > 0) {
    double blk[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) blk[q] = acc[q];
    group_sum<NR>(blk, red, ct, kConsumers, 1);
    int *sflag = const_cast<int *>(flags + kFlagLast);
    if (publish_partials<NR>(blk, a.partials, a.counter, sflag, ct, kConsumers, 1)) {
      double tot[NR];
      reduce_partials<NR>(tot, a.partials, (int)gridDim.x, a.long_dot, a.n_long, 2,
                          a.counter, red, ct, kConsumers, 1);
      if (ct == 0) {
#pragma unroll
        for (int q = 0; q < NR; ++q) a.dot_out[q] = tot[q];
      }
    }
  }
}

// Kernel variants: pipeline depth and CTAs per SM.
struct SpmvVariant {
  int stages;
  int min_blocks;
};
constexpr int kNumSpmvVariants = 4;
constexpr SpmvVariant kSpmvVariants[kNumSpmvVariants] = {{3, 3}, {2, 3}, {2, 4}, {4, 2}};

}  // namespace mlsh
