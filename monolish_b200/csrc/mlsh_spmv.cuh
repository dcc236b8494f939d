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
//    tile's contiguous val[] and col_ind[] ranges into a kStages-deep ring
//    of shared-memory stages with 1-D bulk (TMA) copies that complete on an
//    mbarrier; the other lanes fill the <16-byte ragged ends with plain
//    loads.  HBM sees only long, aligned, fully used bursts.
//  * 8 consumer warps: pass A forms val[j]*x[col[j]] in place over the
//    tile's nonzeros (nonzero-parallel, so the x gathers are balanced and
//    independent; x is read through the read-only path), pass B sums each
//    row of up to kShortRow entries sequentially in one thread (the same
//    order as the reference's row loop, so those rows are bit-identical to
//    it), pass C gives longer rows a whole warp, pass D writes y coalesced
//    and accumulates the fused dots in a fixed per-thread order.
//  * Chunk tiles reduce their products CTA-wide into a per-chunk partial;
//    the last chunk to arrive (atomic counter per long row) sums the
//    partials in chunk order and writes the row.
//  * Every wait on an mbarrier is bounded; on timeout the CTA records
//    MLSH_ERR_TIMEOUT, drains its in-flight copies and exits.
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

template <typename VT>
struct SpmvSmem {
  static constexpr int kValBytes = ((kTileNnz * (int)sizeof(VT) + 16) + 15) & ~15;
  static constexpr int kColBytes = ((kTileNnz * 4 + 16) + 15) & ~15;
  static constexpr int kStageBytes = kValBytes + kColBytes;
  static constexpr int kYsOff = kStages * kStageBytes;
  static constexpr int kBarOff = kYsOff + kTileRows * (int)sizeof(VT) + 16;
  static constexpr int kRedOff = kBarOff + 2 * kStages * 8;
  static constexpr int kFlagOff = kRedOff + 32 * 8;
  static constexpr int kBytes = kFlagOff + 8 * 4;
};

// flags[] in shared memory
constexpr int kFlagProdAbort = 0;
constexpr int kFlagConsAbort = 1;
constexpr int kFlagConsumed = 2;
constexpr int kFlagLast = 3;

template <typename T>
__device__ __forceinline__ int head_elems(const T *base, int idx) {
  return (int)(((uintptr_t)(base + idx) & 15u) / sizeof(T));
}

// Producer side: stage tile `tl` of array `arr` (element type E) into smem
// buffer `dst`, element nnz_begin landing at dst[head].  Returns the bytes
// the bulk copy will deliver (0 if none).  Called by all 32 lanes.
template <typename E>
__device__ __forceinline__ uint32_t stage_range(const E *arr, int nb, int ne,
                                                E *dst, int lane,
                                                uint32_t bar) {
  const uintptr_t b0 = (uintptr_t)(arr + nb);
  const uintptr_t b1 = (uintptr_t)(arr + ne);
  const uintptr_t lo = b0 & ~(uintptr_t)15;
  uintptr_t i0 = (b0 + 15) & ~(uintptr_t)15;
  uintptr_t i1 = b1 & ~(uintptr_t)15;
  const int head = (int)((b0 - lo) / sizeof(E));
  // ragged elements: [nb, e0) and [e1, ne) with e0/e1 the interior bounds
  int e0, e1;
  if (i1 > i0) {
    e0 = nb + (int)((i0 - b0) / sizeof(E));
    e1 = nb + (int)((i1 - b0) / sizeof(E));
  } else {
    e0 = ne;  // everything by plain loads
    e1 = ne;
    i0 = i1 = 0;
  }
  const int nhead = e0 - nb;
  const int ntail = ne - e1;
  if (lane < nhead) dst[head + lane] = arr[nb + lane];
  if (lane >= 16 && lane - 16 < ntail)
    dst[head + (e1 - nb) + (lane - 16)] = arr[e1 + (lane - 16)];
  uint32_t bytes = (uint32_t)(i1 - i0);
  (void)bar;
  return bytes;
}

template <typename VT, typename XT, int M0, int M1>
__global__ void __launch_bounds__(kSpmvThreads, 3)
    spmv_tiles_kernel(const SpmvArgs<VT, XT> a) {
  constexpr int NR = (M0 != kDotNone ? 1 : 0) + (M1 != kDotNone ? 1 : 0);
  using L = SpmvSmem<VT>;
  extern __shared__ __align__(128) unsigned char smem[];
  if (a.done != nullptr && *a.done != 0) return;

  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::kBarOff);
  double *red = reinterpret_cast<double *>(smem + L::kRedOff);
  volatile int *flags = reinterpret_cast<volatile int *>(smem + L::kFlagOff);
  VT *ys = reinterpret_cast<VT *>(smem + L::kYsOff);
  const int tid = threadIdx.x;
  const uint32_t full0 = smem_addr(bars);
  const uint32_t empty0 = smem_addr(bars + kStages);

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int f = 0; f < 8; ++f) flags[f] = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (tid < 32) {
    // ------------------------------------------------------- producer ---
    const int lane = tid;
    int k = 0;
    bool aborted = false;
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++k) {
      const int s = k % kStages;
      if (k >= kStages) {
        int ok = 1;
        if (lane == 0) {
          const uint32_t par = (uint32_t)((k / kStages - 1) & 1);
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
      const Tile tl = a.tiles[t];
      unsigned char *st = smem + s * L::kStageBytes;
      VT *sv = reinterpret_cast<VT *>(st);
      int *sc = reinterpret_cast<int *>(st + L::kValBytes);
      const uint32_t bar = full0 + 8 * s;
      const uint32_t vb = stage_range<VT>(a.val, tl.nnz_begin, tl.nnz_end, sv, lane, bar);
      const uint32_t cb = stage_range<int>(a.col, tl.nnz_begin, tl.nnz_end, sc, lane, bar);
      __threadfence_block();
      __syncwarp();
      if (lane == 0) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, vb + cb);
        if (vb) {
          const uintptr_t i0 = ((uintptr_t)(a.val + tl.nnz_begin) + 15) & ~(uintptr_t)15;
          const uintptr_t lo = (uintptr_t)(a.val + tl.nnz_begin) & ~(uintptr_t)15;
          bulk_g2s(smem_addr(st) + (uint32_t)(i0 - lo), (const void *)i0, vb, bar);
        }
        if (cb) {
          const uintptr_t i0 = ((uintptr_t)(a.col + tl.nnz_begin) + 15) & ~(uintptr_t)15;
          const uintptr_t lo = (uintptr_t)(a.col + tl.nnz_begin) & ~(uintptr_t)15;
          bulk_g2s(smem_addr(st + L::kValBytes) + (uint32_t)(i0 - lo), (const void *)i0, cb, bar);
        }
      }
      __syncwarp();
    }
    const int issued = k;
    // Tail: wait until the consumers have released every issued stage (so
    // no copy is in flight when the CTA exits).  If they aborted, wait for
    // the copies themselves instead.
    if (lane == 0) {
      for (int kk = issued - kStages < 0 ? 0 : issued - kStages; kk < issued; ++kk) {
        const int s = kk % kStages;
        const uint32_t par = (uint32_t)((kk / kStages) & 1);
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
          const int s = kk % kStages;
          mbar_wait_bounded(full0 + 8 * s, (uint32_t)((kk / kStages) & 1), kWaitLimitNs);
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

  int k = 0;
  for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++k) {
    const int s = k % kStages;
    if (ct == 0) {
      if (!mbar_wait_bounded(full0 + 8 * s, (uint32_t)((k / kStages) & 1), kWaitLimitNs)) {
        flags[kFlagConsAbort] = 1;
        atomicExch(a.err, MLSH_ERR_TIMEOUT);
      }
    }
    named_sync(1, kConsumers);
    if (flags[kFlagConsAbort]) break;

    const Tile tl = a.tiles[t];
    const int nb = tl.nnz_begin, ne = tl.nnz_end, nt = ne - nb;
    unsigned char *st = smem + s * L::kStageBytes;
    VT *v = reinterpret_cast<VT *>(st) + head_elems(a.val, nb);
    const int *c = reinterpret_cast<const int *>(st + L::kValBytes) + head_elems(a.col, nb);

    // pass A: products in place
    {
      int cc[kPer];
      XT xx[kPer];
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int j = ct + u * kConsumers;
        cc[u] = (j < nt) ? c[j] : 0;
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

    if (tl.row_end >= 0) {
      // -------------------------------------------------- normal tile ---
      const int rb = tl.row_begin, nrows = tl.row_end - tl.row_begin;
      bool med = false;
      int s0 = 0, s1 = 0;
      if (ct < nrows) {
        s0 = __ldg(a.row_ptr + rb + ct) - nb;
        s1 = __ldg(a.row_ptr + rb + ct + 1) - nb;
        if (s1 - s0 <= kShortRow) {
          VT sum = VT(0);
          for (int j = s0; j < s1; ++j) sum += v[j];
          ys[ct] = sum;
        } else {
          med = true;
        }
      }
      unsigned mask = __ballot_sync(0xffffffffu, med);
      while (mask) {
        const int l = __ffs(mask) - 1;
        mask &= mask - 1;
        const int r0 = __shfl_sync(0xffffffffu, s0, l);
        const int r1 = __shfl_sync(0xffffffffu, s1, l);
        VT sum = VT(0);
        for (int j = r0 + lane; j < r1; j += 32) sum += v[j];
        sum = warp_sum(sum);
        if (lane == 0) ys[warp * 32 + l] = sum;
      }
      named_sync(1, kConsumers);
      if (ct == 0) {
        mbar_arrive(empty0 + 8 * s);
        flags[kFlagConsumed] = k + 1;
      }
      if (ct < nrows) {
        const int r = rb + ct;
        const double sum = (double)ys[ct];
        const XT out = (beta == 0.0) ? (XT)(alpha * sum)
                                     : (XT)(alpha * sum + beta * (double)a.y_in[r]);
        a.y_out[r] = out;
        if constexpr (M0 == kDotW) acc[0] += (double)a.w0[r] * (double)out;
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
      if (ct == 0) {
        mbar_arrive(empty0 + 8 * s);
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

}  // namespace mlsh
