// Matrix set-up on the GPU: COO sorting and merging, COO -> CRS row
// pointers, CRS transposition, and the transposed SpMV built on them.
//
// Reference behaviour restated here:
//   COO::sort(merge)   src/utils/at_insert_sort/at_insert_sort_coo.cpp:119-145
//                      (order by (row, col); merge keeps one entry per
//                      (row, col) with the run's last value)
//   CRS::convert(COO&) src/utils/convert/convert_crs.cpp:9-43
//                      (row pointer of a row-sorted COO)
//   blas::matvec_T     src/blas/matrix/matvec/crs_matvec.hpp:88-98
//                      (y_j = sum over rows i in increasing order of a_ij x_i)
//
// Design: everything is a stable least-significant-digit radix sort of
// (32-bit key, 32-bit entry index) pairs, 8 bits per pass, plus binary
// searches.  Stability makes the results deterministic: a COO sorted by
// column and then by row comes out in (row, col, input position) order, and
// a CRS re-sorted by column keeps the rows of each column in increasing
// order -- the order in which the reference's serial loop accumulates
// y_j, so a transposed row of up to kShortRow entries is summed exactly as
// the reference sums it.
//
// Each radix pass is three launches: a per-tile digit histogram (shared
// atomics), an exclusive scan of the digit-major histogram, and a stable
// scatter in which each 256-item round of a tile ranks its items with
// __match_any_sync (lanes with equal digits), per-warp digit counts in
// shared memory and a per-digit running offset.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "mlsh_core.cuh"

namespace mlsh {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // items per CTA tile
constexpr int kRadix = 256;
constexpr int kSortWarps = kSortThreads / 32;

__device__ __forceinline__ unsigned warp_sum_u(unsigned v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Exclusive scan within the block of one value per thread; returns the
// thread's prefix and writes the block total to *total.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned *warp_tot,
                                                         unsigned *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  unsigned before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const unsigned t = warp_tot[w];
    if (w < warp) before += t;
    all += t;
  }
  *total = all;
  __syncthreads();
  return before + incl - v;
}

// ------------------------------------------------------------------ scan --
// Sum of each kSortTile-item tile.
__global__ void __launch_bounds__(kSortThreads) scan_tile_sums(const unsigned *in, long long n,
                                                               unsigned *sums) {
  __shared__ unsigned wsum[kSortWarps];
  const long long base = (long long)blockIdx.x * kSortTile;
  unsigned s = 0;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const long long i = base + j * kSortThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = warp_sum_u(s);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = 0;
    for (int w = 0; w < kSortWarps; ++w) t += wsum[w];
    sums[blockIdx.x] = t;
  }
}

// Exclusive scan of the tile sums in place (one CTA, chunks of 256 with a
// running carry).
__global__ void __launch_bounds__(kSortThreads) scan_tile_offsets(unsigned *sums, int n_tiles) {
  __shared__ unsigned wtot[kSortWarps];
  unsigned carry = 0;
  for (int c = 0; c < n_tiles; c += kSortThreads) {
    const int i = c + threadIdx.x;
    const unsigned v = i < n_tiles ? sums[i] : 0u;
    unsigned tot;
    const unsigned ex = block_exclusive_scan(v, wtot, &tot);
    if (i < n_tiles) sums[i] = carry + ex;
    carry += tot;
  }
}

// out[i] = tile offset + exclusive prefix within the tile (out may be in).
__global__ void __launch_bounds__(kSortThreads) scan_apply(const unsigned *in, long long n,
                                                           const unsigned *offs, unsigned *out) {
  __shared__ unsigned buf[kSortTile];
  __shared__ unsigned wtot[kSortWarps];
  const long long base = (long long)blockIdx.x * kSortTile;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int k = j * kSortThreads + threadIdx.x;
    buf[k] = base + k < n ? in[base + k] : 0u;
  }
  __syncthreads();
  // thread t owns items [t*16, t*16+16): serial scan, then across threads
  unsigned loc[kSortItems];
  unsigned s = 0;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    loc[j] = s;
    s += buf[threadIdx.x * kSortItems + j];
  }
  unsigned tot;
  const unsigned pre = block_exclusive_scan(s, wtot, &tot) + offs[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) buf[threadIdx.x * kSortItems + j] = pre + loc[j];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const int k = j * kSortThreads + threadIdx.x;
    if (base + k < n) out[base + k] = buf[k];
  }
}

// ----------------------------------------------------------- radix sort --
__global__ void __launch_bounds__(kSortThreads) radix_hist(const unsigned *keys, long long n,
                                                           int shift, unsigned *hist,
                                                           int n_tiles) {
  __shared__ unsigned h[kRadix];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const long long i = base + j * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  hist[(long long)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: items are taken in rounds of 256 in index
// order; within a round a lane's rank among equal digits is the count of
// equal-digit lanes before it in its warp plus those in earlier warps.
__global__ void __launch_bounds__(kSortThreads) radix_scatter(
    const unsigned *keys_in, const unsigned *vals_in, long long n, int shift,
    const unsigned *offs, int n_tiles, unsigned *keys_out, unsigned *vals_out) {
  __shared__ unsigned run[kRadix];
  __shared__ unsigned wcnt[kSortWarps][kRadix];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  run[t] = offs[(long long)t * n_tiles + blockIdx.x];
  const unsigned lt_mask = (1u << lane) - 1u;
  const long long base = (long long)blockIdx.x * kSortTile;
  for (int j = 0; j < kSortItems; ++j) {
    const long long i = base + j * kSortThreads + t;
    const bool valid = i < n;
    const unsigned key = valid ? keys_in[i] : 0u;
    const unsigned val = valid ? vals_in[i] : 0u;
    const unsigned d = valid ? (key >> shift) & (kRadix - 1) : (unsigned)kRadix;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) wcnt[w][t] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned rank = __popc(peers & lt_mask);
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      unsigned pos = run[d] + rank;
      for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    unsigned add = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) add += wcnt[w][t];
    run[t] += add;
    __syncthreads();
  }
}

// ----------------------------------------------------- helper kernels --
__global__ void iota_u32(unsigned *v, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    v[i] = (unsigned)i;
}

__global__ void gather_u32(const unsigned *src, const unsigned *perm, long long n,
                           unsigned *dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

// out[j] = first position whose key is >= j, for j = 0..n_out.
__global__ void lower_bounds(const unsigned *keys, long long n, int n_out, int *out) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j <= n_out;
       j += (long long)gridDim.x * blockDim.x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (keys[mid] < (unsigned)j) lo = mid + 1;
      else hi = mid;
    }
    out[j] = (int)lo;
  }
}

// err |= 1 for an index outside [0, n_rows) x [0, n_cols).
__global__ void coo_range_check(const int *row, const int *col, long long n, int n_rows,
                                int n_cols, int *err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (row[i] < 0 || row[i] >= n_rows || (col && (col[i] < 0 || col[i] >= n_cols)))
      atomicOr(err, 1);
}

// err |= 2 where rows decrease (the COO -> CRS conversion needs row order).
__global__ void rows_sorted_check(const int *row, long long n, int *err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i + 1 < n;
       i += (long long)gridDim.x * blockDim.x)
    if (row[i] > row[i + 1]) atomicOr(err, 2);
}

// Sorted entries into scratch: rows from the sorted keys, columns and
// values through the permutation.
template <typename T>
__global__ void coo_gather(const unsigned *rows_sorted, const unsigned *perm, const int *col,
                           const T *val, long long n, int *row_out, int *col_out, T *val_out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned e = perm[i];
    row_out[i] = (int)rows_sorted[i];
    col_out[i] = col[e];
    val_out[i] = val[e];
  }
}

// flag[i] = 1 where entry i ends its run of equal (row, col).
__global__ void run_end_flags(const int *row, const int *col, long long n, unsigned *flag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    flag[i] = (i + 1 == n || row[i] != row[i + 1] || col[i] != col[i + 1]) ? 1u : 0u;
}

template <typename T>
__global__ void run_compact(const unsigned *flag, const unsigned *pos, const int *row,
                            const int *col, const T *val, long long n, int *row_out,
                            int *col_out, T *val_out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (flag[i]) {
      const unsigned p = pos[i];
      row_out[p] = row[i];
      col_out[p] = col[i];
      val_out[p] = val[i];
    }
}

// Transposed entries: row index of entry perm[k] (binary search in rp) and
// its value.
template <typename T>
__global__ void transpose_fill(const int *rp, int n_rows, const unsigned *perm, long long nnz,
                               const T *val, int *ci_t, T *val_t) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz;
       k += (long long)gridDim.x * blockDim.x) {
    const int e = (int)perm[k];
    int lo = 0, hi = n_rows;  // last row with rp[row] <= e
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(rp + mid) <= e) lo = mid;
      else hi = mid;
    }
    // the last row starting at or before e is never an empty one
    if (ci_t) ci_t[k] = lo;
    val_t[k] = val[e];
  }
}

template <typename T>
__global__ void gather_vals(const unsigned *perm, const T *val, long long n, T *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = val[perm[i]];
}

// ------------------------------------------------------------ host side --
unsigned grid_for(long long n) {
  const long long b = (n + 255) / 256;
  return (unsigned)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}

long long sort_tiles(long long n) { return (n + kSortTile - 1) / kSortTile; }

int bit_length(long long v) {
  int b = 0;
  while (v > 0) {
    ++b;
    v >>= 1;
  }
  return b;
}

// Exclusive scan of n values into out (out may be in); `sums` holds
// sort_tiles(n) entries.
void scan_exclusive(const unsigned *in, unsigned *out, long long n, unsigned *sums,
                    cudaStream_t s) {
  if (n <= 0) return;
  const long long tiles = sort_tiles(n);
  scan_tile_sums<<<(unsigned)tiles, kSortThreads, 0, s>>>(in, n, sums);
  scan_tile_offsets<<<1, kSortThreads, 0, s>>>(sums, (int)tiles);
  scan_apply<<<(unsigned)tiles, kSortThreads, 0, s>>>(in, n, sums, out);
}

// Radix-sort scratch for n pairs: two key and two index buffers, the
// digit histogram and the scan's tile sums, in one pool allocation.
struct SortScratch {
  void *base = nullptr;
  unsigned *k[2] = {nullptr, nullptr};
  unsigned *v[2] = {nullptr, nullptr};
  unsigned *hist = nullptr;
  unsigned *sums = nullptr;
  char *extra = nullptr;  // caller-sized tail
  cudaStream_t s = nullptr;

  int alloc(long long n, size_t extra_bytes, cudaStream_t stream) {
    s = stream;
    const long long tiles = sort_tiles(n);
    const size_t vec = ((size_t)n * 4 + 255) / 256 * 256;
    const size_t hist_b = ((size_t)kRadix * tiles * 4 + 255) / 256 * 256;
    const size_t sums_b = ((size_t)(tiles + 1) * 4 + 255) / 256 * 256;
    const size_t total = 4 * vec + hist_b + sums_b + extra_bytes;
    if (pool_alloc(&base, total, s) != cudaSuccess) {
      cudaGetLastError();
      return MLSH_ERR_OOM;
    }
    char *p = static_cast<char *>(base);
    k[0] = reinterpret_cast<unsigned *>(p);
    v[0] = reinterpret_cast<unsigned *>(p + vec);
    k[1] = reinterpret_cast<unsigned *>(p + 2 * vec);
    v[1] = reinterpret_cast<unsigned *>(p + 3 * vec);
    hist = reinterpret_cast<unsigned *>(p + 4 * vec);
    sums = reinterpret_cast<unsigned *>(p + 4 * vec + hist_b);
    extra = p + 4 * vec + hist_b + sums_b;
    return MLSH_SUCCESS;
  }
  ~SortScratch() {
    if (base) {
      cudaStreamSynchronize(s);
      pool_free(base, s);
    }
  }
};

// Stable sort of the pairs in (k[src], v[src]) by the low `bits` bits of
// the keys; returns the buffer index that holds the result.
int radix_sort_pairs(SortScratch &w, int src, long long n, int bits) {
  const long long tiles = sort_tiles(n);
  for (int shift = 0; shift < bits; shift += 8) {
    const int dst = src ^ 1;
    radix_hist<<<(unsigned)tiles, kSortThreads, 0, w.s>>>(w.k[src], n, shift, w.hist,
                                                          (int)tiles);
    scan_exclusive(w.hist, w.hist, (long long)kRadix * tiles, w.sums, w.s);
    radix_scatter<<<(unsigned)tiles, kSortThreads, 0, w.s>>>(w.k[src], w.v[src], n, shift,
                                                             w.hist, (int)tiles, w.k[dst],
                                                             w.v[dst]);
    src = dst;
  }
  return src;
}

// Reads back the device error word (synchronizes the stream).
int read_flag(const int *d_flag, cudaStream_t s, int *out) {
  MLSH_CUDA_TRY(cudaMemcpyAsync(out, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  return MLSH_SUCCESS;
}

}  // namespace
}  // namespace mlsh

namespace mlsh {
namespace {

template <typename T>
void coo_gather_t(const unsigned *rows, const unsigned *perm, const int *col, const void *val,
                  long long n, int *row_out, int *col_out, void *val_out, cudaStream_t s) {
  coo_gather<T><<<grid_for(n), 256, 0, s>>>(rows, perm, col, static_cast<const T *>(val), n,
                                            row_out, col_out, static_cast<T *>(val_out));
}

template <typename T>
void run_compact_t(const unsigned *flag, const unsigned *pos, const int *row, const int *col,
                   const void *val, long long n, int *row_out, int *col_out, void *val_out,
                   cudaStream_t s) {
  run_compact<T><<<grid_for(n), 256, 0, s>>>(flag, pos, row, col, static_cast<const T *>(val),
                                             n, row_out, col_out, static_cast<T *>(val_out));
}

}  // namespace

// A^T of an n_rows x n_cols CRS into (rp_t, ci_t, val_t); the entry
// permutation (position in A of each entry of A^T) into perm_out if given.
int transpose_build(Handle &h, int n_rows, int n_cols, int nnz, const int *rp, const int *ci,
                    const void *val, int dtype, int *rp_t, int *ci_t, void *val_t,
                    unsigned *perm_out) {
  cudaStream_t s = h.stream;
  if (nnz == 0) {
    MLSH_CUDA_TRY(cudaMemsetAsync(rp_t, 0, sizeof(int) * ((size_t)n_cols + 1), s));
    MLSH_CUDA_TRY(cudaStreamSynchronize(s));
    return MLSH_SUCCESS;
  }
  SortScratch w;
  int st = w.alloc(nnz, 256, s);
  if (st != MLSH_SUCCESS) return st;
  int *d_err = reinterpret_cast<int *>(w.extra);
  MLSH_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  coo_range_check<<<grid_for(nnz), 256, 0, s>>>(ci, nullptr, nnz, n_cols, 0, d_err);
  int err = 0;
  st = read_flag(d_err, s, &err);
  if (st != MLSH_SUCCESS) return st;
  if (err) return MLSH_ERR_INVALID_CSR;
  MLSH_CUDA_TRY(cudaMemcpyAsync(w.k[0], ci, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToDevice,
                                s));
  iota_u32<<<grid_for(nnz), 256, 0, s>>>(w.v[0], nnz);
  const int r = radix_sort_pairs(w, 0, nnz, bit_length((long long)n_cols - 1));
  lower_bounds<<<grid_for((long long)n_cols + 1), 256, 0, s>>>(w.k[r], nnz, n_cols, rp_t);
  if (dtype == MLSH_F64)
    transpose_fill<double><<<grid_for(nnz), 256, 0, s>>>(
        rp, n_rows, w.v[r], nnz, static_cast<const double *>(val), ci_t,
        static_cast<double *>(val_t));
  else
    transpose_fill<float><<<grid_for(nnz), 256, 0, s>>>(
        rp, n_rows, w.v[r], nnz, static_cast<const float *>(val), ci_t,
        static_cast<float *>(val_t));
  if (perm_out)
    MLSH_CUDA_TRY(cudaMemcpyAsync(perm_out, w.v[r], sizeof(unsigned) * (size_t)nnz,
                                  cudaMemcpyDeviceToDevice, s));
  MLSH_CUDA_TRY(cudaGetLastError());
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  return MLSH_SUCCESS;
}

namespace {

// The transpose kept with a plan for mlsh_spmv_transpose.
struct TransposeCache {
  mlsh_csr_plan plan_t = nullptr;
  int *rp_t = nullptr, *ci_t = nullptr;
  void *val_t = nullptr;
  unsigned *perm = nullptr;
  bool vals_valid = false;
  cudaStream_t s = nullptr;  // stream of the buffers' allocation
};

void free_cache(TransposeCache *c) {
  if (!c) return;
  if (c->plan_t) mlsh_csr_plan_destroy(c->plan_t);
  cudaStreamSynchronize(c->s);
  for (void *d : {(void *)c->rp_t, (void *)c->ci_t, c->val_t, (void *)c->perm})
    pool_free(d, c->s);
  cudaStreamSynchronize(c->s);
  delete c;
}

int ensure_transpose(mlsh_handle hs, CsrPlan &p, TransposeCache **out) {
  Handle &h = hs->h;
  auto *c = static_cast<TransposeCache *>(p.transpose);
  const size_t esz = (size_t)dtype_size(p.dtype);
  if (c && c->vals_valid) {
    *out = c;
    return MLSH_SUCCESS;
  }
  if (c) {  // values changed: same structure, gather the new values
    if (p.nnz > 0) {
      if (p.dtype == MLSH_F64)
        gather_vals<double><<<grid_for(p.nnz), 256, 0, h.stream>>>(
            c->perm, static_cast<const double *>(p.val), p.nnz, static_cast<double *>(c->val_t));
      else
        gather_vals<float><<<grid_for(p.nnz), 256, 0, h.stream>>>(
            c->perm, static_cast<const float *>(p.val), p.nnz, static_cast<float *>(c->val_t));
      MLSH_CUDA_TRY(cudaGetLastError());
    }
    mlsh_csr_plan_values_changed(c->plan_t);
    c->vals_valid = true;
    *out = c;
    return MLSH_SUCCESS;
  }
  c = new (std::nothrow) TransposeCache();
  if (!c) return MLSH_ERR_OOM;
  c->s = h.stream;
  const size_t nnz1 = (size_t)std::max(p.nnz, 1);
  if (pool_alloc(&c->rp_t, sizeof(int) * ((size_t)p.n_cols + 1), c->s) != cudaSuccess ||
      pool_alloc(&c->ci_t, sizeof(int) * nnz1, c->s) != cudaSuccess ||
      pool_alloc(&c->val_t, esz * nnz1, c->s) != cudaSuccess ||
      pool_alloc(&c->perm, sizeof(unsigned) * nnz1, c->s) != cudaSuccess) {
    cudaGetLastError();
    free_cache(c);
    return MLSH_ERR_OOM;
  }
  int st = transpose_build(h, p.n_rows, p.n_cols, p.nnz, p.row_ptr, p.col_ind, p.val, p.dtype,
                           c->rp_t, c->ci_t, c->val_t, c->perm);
  std::vector<int> host_rp((size_t)p.n_cols + 1);
  if (st == MLSH_SUCCESS &&
      cudaMemcpy(host_rp.data(), c->rp_t, sizeof(int) * host_rp.size(),
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    st = MLSH_ERR_CUDA;
  if (st == MLSH_SUCCESS)
    st = mlsh_csr_plan_create(hs, p.n_cols, p.n_rows, p.nnz, c->rp_t, c->ci_t, c->val_t,
                              p.dtype, host_rp.data(), 0, &c->plan_t);
  if (st != MLSH_SUCCESS) {
    free_cache(c);
    return st;
  }
  c->plan_t->p.variant = p.variant;
  c->vals_valid = true;
  p.transpose = c;
  *out = c;
  return MLSH_SUCCESS;
}

}  // namespace

void transpose_release(CsrPlan &p) {
  free_cache(static_cast<TransposeCache *>(p.transpose));
  p.transpose = nullptr;
}

void transpose_invalidate(CsrPlan &p) {
  auto *c = static_cast<TransposeCache *>(p.transpose);
  if (c) c->vals_valid = false;
}

}  // namespace mlsh

using namespace mlsh;

extern "C" {

int mlsh_coo_sort(mlsh_handle hs, int n_rows, int n_cols, int64_t nnz, int *d_row, int *d_col,
                  void *d_val, int dtype, int merge, int64_t *new_nnz) {
  if (!hs || !new_nnz || n_rows < 0 || n_cols < 0 || nnz < 0 || nnz > INT32_MAX ||
      dtype_size(dtype) == 0 || (nnz > 0 && (!d_row || !d_col || !d_val)))
    return MLSH_ERR_INVALID_ARG;
  *new_nnz = 0;
  if (nnz == 0) return MLSH_SUCCESS;
  Handle &h = hs->h;
  cudaStream_t s = h.stream;
  const long long n = nnz;
  const size_t esz = (size_t)dtype_size(dtype);
  const size_t vec4 = ((size_t)n * 4 + 255) / 256 * 256;
  const size_t vecv = ((size_t)n * esz + 255) / 256 * 256;
  // extra: error word, sorted rows/cols/values, run flags and positions
  SortScratch w;
  int st = w.alloc(n, 256 + 4 * vec4 + vecv, s);
  if (st != MLSH_SUCCESS) return st;
  int *d_err = reinterpret_cast<int *>(w.extra);
  int *t_row = reinterpret_cast<int *>(w.extra + 256);
  int *t_col = reinterpret_cast<int *>(w.extra + 256 + vec4);
  unsigned *flag = reinterpret_cast<unsigned *>(w.extra + 256 + 2 * vec4);
  unsigned *pos = reinterpret_cast<unsigned *>(w.extra + 256 + 3 * vec4);
  void *t_val = w.extra + 256 + 4 * vec4;
  MLSH_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  coo_range_check<<<grid_for(n), 256, 0, s>>>(d_row, d_col, n, n_rows, n_cols, d_err);
  int err = 0;
  st = read_flag(d_err, s, &err);
  if (st != MLSH_SUCCESS) return st;
  if (err) return MLSH_ERR_INVALID_ARG;
  // stable by column, then stable by row: (row, col, input position) order
  MLSH_CUDA_TRY(cudaMemcpyAsync(w.k[0], d_col, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
  iota_u32<<<grid_for(n), 256, 0, s>>>(w.v[0], n);
  int r = radix_sort_pairs(w, 0, n, bit_length((long long)n_cols - 1));
  const int o = r ^ 1;
  gather_u32<<<grid_for(n), 256, 0, s>>>(reinterpret_cast<const unsigned *>(d_row), w.v[r], n,
                                         w.k[o]);
  // rows in k[o] with the permutation in v[r]: make them one pair
  std::swap(w.v[r], w.v[o]);
  r = radix_sort_pairs(w, o, n, bit_length((long long)n_rows - 1));
  if (esz == 8)
    coo_gather_t<double>(w.k[r], w.v[r], d_col, d_val, n, t_row, t_col, t_val, s);
  else
    coo_gather_t<float>(w.k[r], w.v[r], d_col, d_val, n, t_row, t_col, t_val, s);
  long long out_n = n;
  if (!merge) {
    MLSH_CUDA_TRY(cudaMemcpyAsync(d_row, t_row, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    MLSH_CUDA_TRY(cudaMemcpyAsync(d_col, t_col, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    MLSH_CUDA_TRY(cudaMemcpyAsync(d_val, t_val, esz * n, cudaMemcpyDeviceToDevice, s));
  } else {
    run_end_flags<<<grid_for(n), 256, 0, s>>>(t_row, t_col, n, flag);
    scan_exclusive(flag, pos, n, w.sums, s);
    unsigned last[2] = {0, 0};
    MLSH_CUDA_TRY(cudaMemcpyAsync(&last[0], pos + n - 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                  s));
    MLSH_CUDA_TRY(cudaMemcpyAsync(&last[1], flag + n - 1, sizeof(unsigned),
                                  cudaMemcpyDeviceToHost, s));
    if (esz == 8)
      run_compact_t<double>(flag, pos, t_row, t_col, t_val, n, d_row, d_col, d_val, s);
    else
      run_compact_t<float>(flag, pos, t_row, t_col, t_val, n, d_row, d_col, d_val, s);
    MLSH_CUDA_TRY(cudaStreamSynchronize(s));
    out_n = (long long)last[0] + last[1];
  }
  MLSH_CUDA_TRY(cudaGetLastError());
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  *new_nnz = out_n;
  return MLSH_SUCCESS;
}

int mlsh_coo_to_csr(mlsh_handle hs, int n_rows, int64_t nnz, const int *d_row, int *d_row_ptr) {
  if (!hs || n_rows < 0 || nnz < 0 || nnz > INT32_MAX || !d_row_ptr || (nnz > 0 && !d_row))
    return MLSH_ERR_INVALID_ARG;
  cudaStream_t s = hs->h.stream;
  if (nnz > 0) {
    int *d_err = nullptr;
    if (pool_alloc(&d_err, sizeof(int), s) != cudaSuccess) {
      cudaGetLastError();
      return MLSH_ERR_OOM;
    }
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    coo_range_check<<<grid_for(nnz), 256, 0, s>>>(d_row, nullptr, nnz, n_rows, 0, d_err);
    rows_sorted_check<<<grid_for(nnz), 256, 0, s>>>(d_row, nnz, d_err);
    int err = 0;
    const int st = read_flag(d_err, s, &err);
    pool_free(d_err, s);
    if (st != MLSH_SUCCESS) return st;
    if (err) return MLSH_ERR_INVALID_CSR;
  }
  lower_bounds<<<grid_for((long long)n_rows + 1), 256, 0, s>>>(
      reinterpret_cast<const unsigned *>(d_row), nnz, n_rows, d_row_ptr);
  MLSH_CUDA_TRY(cudaGetLastError());
  MLSH_CUDA_TRY(cudaStreamSynchronize(s));
  return MLSH_SUCCESS;
}

int mlsh_csr_transpose(mlsh_handle hs, int n_rows, int n_cols, int nnz, const int *d_rp,
                       const int *d_ci, const void *d_val, int dtype, int *d_rp_t, int *d_ci_t,
                       void *d_val_t) {
  if (!hs || n_rows < 0 || n_cols < 0 || nnz < 0 || dtype_size(dtype) == 0 || !d_rp_t ||
      (nnz > 0 && (!d_rp || !d_ci || !d_val || !d_ci_t || !d_val_t)))
    return MLSH_ERR_INVALID_ARG;
  return transpose_build(hs->h, n_rows, n_cols, nnz, d_rp, d_ci, d_val, dtype, d_rp_t, d_ci_t,
                         d_val_t, nullptr);
}

int mlsh_spmv_transpose(mlsh_handle hs, mlsh_csr_plan ps, double alpha, const void *x,
                        double beta, void *y) {
  if (!hs || !ps || !y || (ps->p.n_rows > 0 && !x)) return MLSH_ERR_INVALID_ARG;
  TransposeCache *c = nullptr;
  const int st = ensure_transpose(hs, ps->p, &c);
  if (st != MLSH_SUCCESS) return st;
  return mlsh_spmv(hs, c->plan_t, alpha, x, beta, y);
}

}  // extern "C"
