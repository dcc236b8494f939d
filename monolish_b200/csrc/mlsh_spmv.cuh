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
//    tile's contiguous val[] and col_ind[] ranges (rounded out to 16-byte
//    boundaries) into a STAGES-deep ring of shared-memory stages with 1-D
//    bulk (TMA) copies that complete on an mbarrier.  HBM sees only long,
//    aligned, fully used bursts, and the copies carry an L2 evict-first
//    policy so the once-read matrix does not push the gathered x out of L2.
//  * 8 consumer warps, each owning 32 rows of the tile and working on its
//    own: it releases the stage itself and, for plain SpMV, also waits on
//    the stage's "full" mbarrier itself, so warps run ahead of one another
//    within the stages in flight (no CTA barrier per tile; only chunk tiles
//    bring them together; the fused-dot launches keep one barrier per tile):
//      rows of up to the plan's short-row limit (8, 16 or 32 entries,
//              picked by the autotuner): one thread each, gathering x 8
//              entries at a time and summing in row order with separately
//              rounded products (the reference's loop, so those rows are
//              bit-identical to it);
//      longer rows: the whole warp, one such row after another (lane-
//              strided partial sums, then an xor tree) -- deterministic;
//      then y is written coalesced and the fused dots accumulate in a
//      fixed per-thread order.  Each thread's row bounds, dot weight and
//      the tile's column base for the next tile are fetched one tile ahead.
//  * Chunk tiles reduce their products CTA-wide into a per-chunk partial;
//    the last chunk to arrive (atomic counter per long row) sums the
//    partials in chunk order and writes the row.
//  * Every wait on an mbarrier is bounded; on timeout the CTA records
//    MLSH_ERR_TIMEOUT, drains its in-flight copies and exits (a consumer
//    warp that gave up keeps walking the tiles only to take part in the
//    chunk tiles' barriers).
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
  int short_max;    // rows up to this length: one thread, in row order
};

template <typename VT, int STAGES, int CSZ = 4>
struct SpmvSmem {
  // a tile's range rounded out to 16-byte boundaries: at most 32 extra bytes
  static constexpr int kValBytes = ((kTileNnz * (int)sizeof(VT) + 32) + 15) & ~15;
  static constexpr int kColBytes = ((kTileNnz * CSZ + 32) + 15) & ~15;
  static constexpr int kStageBytes = kValBytes + kColBytes;
  static constexpr int kBarOff = STAGES * kStageBytes;
  static constexpr int kRedOff = kBarOff + 2 * STAGES * 8;
  static constexpr int kFlagOff = kRedOff + 32 * 8;
  static constexpr int kBytes = kFlagOff + 16 * 4;
};

// flags[] in shared memory
constexpr int kFlagProdAbort = 0;
constexpr int kFlagConsAbort = 1;
constexpr int kFlagLast = 3;
constexpr int kFlagWarpDone = 4;  // 8 slots: tiles each consumer warp has consumed

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
  pdl_wait();
  pdl_launch_dependents();
  if (a.done != nullptr && *a.done != 0) return;

  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::kBarOff);
  double *red = reinterpret_cast<double *>(smem + L::kRedOff);
  volatile int *flags = reinterpret_cast<volatile int *>(smem + L::kFlagOff);
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
          for (uint32_t it = 1;; ++it) {
            if (mbar_try_wait(empty0 + 8 * s, par)) { ok = 1; break; }
            if ((it & 63u) == 0 && flags[kFlagConsAbort]) break;
            if ((it & 1023u) == 0 && global_timer_ns() - t0 > kWaitLimitNs) {
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
        for (uint32_t it = 1;; ++it) {
          if (mbar_try_wait(empty0 + 8 * s, par)) { ok = true; break; }
          if ((it & 63u) == 0 && flags[kFlagConsAbort]) break;
          if ((it & 1023u) == 0 && global_timer_ns() - t0 > kWaitLimitNs) break;
        }
        if (!ok) { aborted = true; break; }
      }
      if (aborted) {
        atomicExch(a.err, MLSH_ERR_TIMEOUT);
        // progress of the slowest consumer warp (with fused dots the warps
        // move together and only the first one reports)
        int consumed = issued;
        for (int w = 0; w < (NR == 0 ? kConsumers / 32 : 1); ++w)
          consumed = min(consumed, (int)flags[kFlagWarpDone + w]);
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

  // Plain SpMV (no fused dots): each warp waits for a stage on its own and
  // releases it on its own, so warps run ahead of one another within the
  // stages in flight, and only a chunk tile (a CTA-wide sum) brings them
  // together.  A warp whose wait gives up stops computing but keeps walking
  // the tiles so that it still takes part in every chunk tile's barrier.
  int k = 0;
  int nchunk = 0;  // chunk tiles met so far (the same count in every warp)
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
    if constexpr (NR == 0) {
      int ok = 1;
      if (lane == 0) {
        // once any warp has given up, the flag sends every warp down the
        // walking path at its next tile
        ok = flags[kFlagConsAbort] == 0 &&
             mbar_wait_bounded(full0 + 8 * s, (uint32_t)((k / STAGES) & 1), kWaitLimitNs);
        if (!ok && flags[kFlagConsAbort] == 0) {
          flags[kFlagConsAbort] = 1;
          atomicExch(a.err, MLSH_ERR_TIMEOUT);
        }
      }
      if (__shfl_sync(0xffffffffu, ok, 0) == 0) {
        tl_c = tl_n;
        if (!normal) {
          named_sync(1, kConsumers);  // the chunk tile's barrier
          ++nchunk;
        }
        continue;
      }
    } else {
      // with fused dots (the solvers' launches, at the register limit) the
      // consumers start each tile together: one thread waits, a CTA-wide
      // named barrier releases all
      if (ct == 0) {
        if (!mbar_wait_bounded(full0 + 8 * s, (uint32_t)((k / STAGES) & 1), kWaitLimitNs)) {
          flags[kFlagConsAbort] = 1;
          atomicExch(a.err, MLSH_ERR_TIMEOUT);
        }
      }
      named_sync(1, kConsumers);
      if (flags[kFlagConsAbort]) break;
    }

    const int nb = tl.nnz_begin, ne = tl.nnz_end, nt = ne - nb;
    unsigned char *st = smem + s * L::kStageBytes;
    const VT *v = reinterpret_cast<const VT *>(st) + head_elems(a.val, nb);
    const uint16_t *c16 = reinterpret_cast<const uint16_t *>(st + L::kValBytes) +
                          (C16 ? head_elems(a.col16, nb) : 0);
    const int *c32 = reinterpret_cast<const int *>(st + L::kValBytes) +
                     (C16 ? 0 : head_elems(a.col, nb));
    // column of the tile's j-th staged entry
    auto col_at = [&](int j) -> int {
      if constexpr (C16) return col_base + (int)c16[j];
      else return c32[j];
    };
    // the next tile's per-thread values, fetched while this tile computes
    auto prefetch_next = [&]() {
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
    };

    if (normal) {
      // Each warp handles its 32 rows on its own (no CTA barrier):
      //  * rows of up to the plan's short-row limit (8, 16 or 32 entries):
      //    one thread each, gathering and summing in row order with
      //    separately rounded products -- the reference's loop, so these
      //    rows are bit-identical to it;
      //  * longer rows: the whole warp, one row after another (lane-strided
      //    partial sums, then an xor tree), the owning thread keeps the sum.
      VT sum = VT(0);
      const int s0 = g0 - nb, len = g1 - g0;
      const int smax = a.short_max;
      if (ct < nrows && len <= smax) {
        // kShortRow gathers in flight at a time; the sum stays in row order
        for (int u0 = 0; u0 < len; u0 += kShortRow) {
          XT xx[kShortRow];
#pragma unroll
          for (int u = 0; u < kShortRow; ++u)
            if (u0 + u < len) xx[u] = __ldg(a.x + col_at(s0 + u0 + u));
#pragma unroll
          for (int u = 0; u < kShortRow; ++u)
            if (u0 + u < len) sum = spmv_add_rn(sum, spmv_mul_rn(v[s0 + u0 + u], (VT)xx[u]));
        }
      }
      prefetch_next();
      unsigned lm = __ballot_sync(0xffffffffu, ct < nrows && len > smax);
      while (lm) {
        const int src = __ffs(lm) - 1;
        lm &= lm - 1;
        const int ls = __shfl_sync(0xffffffffu, s0, src);
        const int le = ls + __shfl_sync(0xffffffffu, len, src);
        VT part = VT(0);
        int j = ls + lane;
        for (; j + 96 < le; j += 128) {
          const XT x0 = __ldg(a.x + col_at(j)), x1 = __ldg(a.x + col_at(j + 32)),
                   x2 = __ldg(a.x + col_at(j + 64)), x3 = __ldg(a.x + col_at(j + 96));
          part = spmv_add_rn(part, spmv_mul_rn(v[j], (VT)x0));
          part = spmv_add_rn(part, spmv_mul_rn(v[j + 32], (VT)x1));
          part = spmv_add_rn(part, spmv_mul_rn(v[j + 64], (VT)x2));
          part = spmv_add_rn(part, spmv_mul_rn(v[j + 96], (VT)x3));
        }
        for (; j < le; j += 32) part = spmv_add_rn(part, spmv_mul_rn(v[j], (VT)__ldg(a.x + col_at(j))));
        part = warp_sum(part);
        if (lane == src) sum = part;
      }
      // this warp is done with the stage
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(empty0 + 8 * s);
        if (NR == 0 || warp == 0) flags[kFlagWarpDone + warp] = k + 1;
      }
      // ----------------------------------------------------- y and dots
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
    } else {
      // --------------------------------------------- chunk of a long row ---
      VT part = VT(0);
      for (int j = ct; j < nt; j += kConsumers)
        part = spmv_add_rn(part, spmv_mul_rn(v[j], (VT)__ldg(a.x + col_at(j))));
      prefetch_next();
      part = warp_sum(part);
      // slots 16..31 of red, apart from the slots the closing dot reduction
      // writes; with independent warps double-buffered by chunk count (a
      // warp can be at most one chunk tile ahead of the thread that reads
      // the sums: it cannot pass the next chunk's barrier before it)
      double *cred = red + 16;
      if constexpr (NR == 0) {
        cred += (nchunk & 1) * (kConsumers / 32);
        ++nchunk;
      }
      if (lane == 0) cred[warp] = (double)part;
      named_sync(1, kConsumers);
      if (lane == 0) {
        mbar_arrive(empty0 + 8 * s);
        if (NR == 0 || warp == 0) flags[kFlagWarpDone + warp] = k + 1;
      }
      if (ct == 0) {
        double tot = 0.0;
        for (int w = 0; w < kConsumers / 32; ++w) tot += cred[w];
        const int li = -tl.row_end - 1;
        const int row = tl.row_begin;
        bool last = true;
        double sum = tot;
        if (tl.pad[0] > 1) {
          // several chunks: the last one to arrive sums them in chunk order
          const LongRow lr = a.longs[li];
          const int slot = lr.first_slot + (nb - __ldg(a.row_ptr + row)) / kTileNnz;
          a.chunk_part[slot] = tot;
          __threadfence();
          const unsigned prev = atomicAdd(a.long_cnt + li, 1u);
          last = prev == (unsigned)(lr.n_chunks - 1);
          if (last) {
            __threadfence();
            sum = 0.0;
            for (int q = 0; q < lr.n_chunks; ++q)
              sum += __ldcg(a.chunk_part + lr.first_slot + q);
            a.long_cnt[li] = 0u;
          }
        }
        if (last) {
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
constexpr int kNumSpmvVariants = 5;
constexpr SpmvVariant kSpmvVariants[kNumSpmvVariants] = {{3, 3}, {2, 3}, {2, 4}, {4, 2}, {3, 4}};

}  // namespace mlsh
