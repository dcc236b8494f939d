// Handle, CRS plan, SpMV and vector-BLAS entry points of the C ABI
// (declared in include/mlsh.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "mlsh_core.cuh"

namespace mlsh {

namespace {
thread_local char g_last_error[256] = "";
}

void set_last_error(const char *where, cudaError_t e) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s", where,
                cudaGetErrorString(e));
}

void set_last_error_text(const char *text) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", text);
}

// --------------------------------------------------------------- tiling --
void build_tiles(const int *rp, int n_rows, std::vector<Tile> &tiles,
                 std::vector<LongRow> &longs, int &n_chunks) {
  tiles.clear();
  longs.clear();
  n_chunks = 0;
  int r = 0;
  while (r < n_rows) {
    const int len = rp[r + 1] - rp[r];
    if (len > kLongRow) {
      const int li = (int)longs.size();
      const int nch = (len + kTileNnz - 1) / kTileNnz;
      longs.push_back(LongRow{r, n_chunks, nch, 0});
      for (int c = 0; c < nch; ++c) {
        const int b = rp[r] + c * kTileNnz;
        const int e = std::min(b + kTileNnz, rp[r + 1]);
        tiles.push_back(Tile{r, -(li + 1), b, e, 0, {nch, 0, 0}});
      }
      n_chunks += nch;
      ++r;
      continue;
    }
    const int rb = r;
    int nnz = 0, longest = 0;
    while (r < n_rows && r - rb < kTileRows) {
      const int l = rp[r + 1] - rp[r];
      if (l > kLongRow || nnz + l > kTileNnz) break;
      nnz += l;
      longest = std::max(longest, l);
      ++r;
    }
    tiles.push_back(Tile{rb, r, rp[rb], rp[r], longest <= kShortRow ? 1 : 0, {0, 0, 0}});
  }
}

// Every (type, dot modes, variant) instantiation of the SpMV kernel.
template <typename VT, int M0, int M1, int V, bool C16 = false>
static constexpr auto spmv_kernel_ptr() {
  return spmv_tiles_kernel<VT, VT, M0, M1, kSpmvVariants[V].stages, kSpmvVariants[V].min_blocks,
                           C16>;
}

template <typename VT, int V, bool C16 = false>
static constexpr int spmv_smem_bytes() {
  return SpmvSmem<VT, kSpmvVariants[V].stages, C16 ? 2 : 4>::kBytes;
}

template <typename VT, int M0, int M1, int V, bool C16 = false>
static int set_spmv_smem_one() {
  const cudaError_t e = cudaFuncSetAttribute(spmv_kernel_ptr<VT, M0, M1, V, C16>(),
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             spmv_smem_bytes<VT, V, C16>());
  if (e != cudaSuccess) {
    set_last_error("cudaFuncSetAttribute(spmv)", e);
    return MLSH_ERR_CUDA;
  }
  return MLSH_SUCCESS;
}

template <typename VT, int M0, int M1>
static int set_spmv_smem() {
  int s = set_spmv_smem_one<VT, M0, M1, 0>();
  if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 1>();
  if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 2>();
  if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 3>();
  if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 4>();
  if constexpr (sizeof(VT) == 4) {
    if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 0, true>();
    if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 1, true>();
    if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 2, true>();
    if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 3, true>();
    if (s == MLSH_SUCCESS) s = set_spmv_smem_one<VT, M0, M1, 4, true>();
  }
  return s;
}

int init_kernel_attributes() {
  static std::once_flag once;
  static int status = MLSH_SUCCESS;
  std::call_once(once, [] {
    int s = MLSH_SUCCESS;
#define MLSH_SET(VT, A, B) \
  if (s == MLSH_SUCCESS) s = set_spmv_smem<VT, A, B>();
    MLSH_SET(double, kDotNone, kDotNone)
    MLSH_SET(double, kDotW, kDotNone)
    MLSH_SET(double, kDotW, kDotSelf)
    MLSH_SET(double, kDotSelf, kDotNone)
    MLSH_SET(float, kDotNone, kDotNone)
    MLSH_SET(float, kDotW, kDotNone)
    MLSH_SET(float, kDotW, kDotSelf)
    MLSH_SET(float, kDotSelf, kDotNone)
#undef MLSH_SET
    status = s;
  });
  return status;
}

template <typename VT, int V>
static int spmv_grid_one(int n_tiles, int num_sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, spmv_kernel_ptr<VT, kDotNone, kDotNone, V>(), kSpmvThreads,
          spmv_smem_bytes<VT, V>()) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  int g = per_sm * num_sms;
  if (g > n_tiles) g = n_tiles;
  if (g > kMaxPartialBlocks) g = kMaxPartialBlocks;
  if (g < 1) g = 1;
  return g;
}

template <typename VT>
static void spmv_grids(int n_tiles, int num_sms, int *grid) {
  grid[0] = spmv_grid_one<VT, 0>(n_tiles, num_sms);
  grid[1] = spmv_grid_one<VT, 1>(n_tiles, num_sms);
  grid[2] = spmv_grid_one<VT, 2>(n_tiles, num_sms);
  grid[3] = spmv_grid_one<VT, 3>(n_tiles, num_sms);
  grid[4] = spmv_grid_one<VT, 4>(n_tiles, num_sms);
}

// ------------------------------------------------------- SpMV launcher --
template <typename VT, int M0, int M1>
cudaError_t launch_spmv_t(const CsrPlan &p, const Handle &h, double alpha,
                          const VT *x, double beta, const VT *y_in, VT *y_out,
                          const VT *w0, const VT *w1, double *dot_out,
                          const int *done, cudaStream_t stream) {
  SpmvArgs<VT, VT> a;
  a.row_ptr = p.row_ptr;
  a.col = p.col_ind;
  a.col16 = p.col16;
  a.tile_base = p.tile_base;
  a.val = static_cast<const VT *>(p.val);
  a.tiles = p.tiles;
  a.n_tiles = p.n_tiles;
  a.n_long = p.n_long;
  a.longs = p.longs;
  a.chunk_part = p.chunk_part;
  a.long_cnt = p.long_cnt;
  a.long_dot = p.long_dot;
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
  a.short_max = p.short_max;
  int v = p.variant;
  // FP64 with two fused dots does not fit 4 CTAs per SM (56 registers: it
  // spills); it runs the same pipeline depth at 3 CTAs per SM instead
  if constexpr (sizeof(VT) == 8 && M0 != kDotNone && M1 != kDotNone) {
    static_assert(kSpmvVariants[2].min_blocks == 4 && kSpmvVariants[1].min_blocks == 3 &&
                      kSpmvVariants[1].stages == kSpmvVariants[2].stages,
                  "variant 1 is variant 2 at 3 CTAs per SM");
    static_assert(kSpmvVariants[4].min_blocks == 4 && kSpmvVariants[0].min_blocks == 3 &&
                      kSpmvVariants[0].stages == kSpmvVariants[4].stages,
                  "variant 0 is variant 4 at 3 CTAs per SM");
    if (v == 2) v = 1;
    if (v == 4) v = 0;
  }
  const int g = p.spmv_grid[v];
  cudaError_t e = cudaSuccess;
  if constexpr (sizeof(VT) == 4) {
    if (p.slots != nullptr)
      return launch_spmv_slots<M0, M1>(p, h, alpha, x, beta, y_in, y_out, w0, w1, dot_out,
                                       done, stream);
    if (p.col16 != nullptr) {
      switch (v) {
        case 1:
          e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 1, true>(), g, kSpmvThreads,
                               spmv_smem_bytes<VT, 1, true>(), stream, a);
          break;
        case 2:
          e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 2, true>(), g, kSpmvThreads,
                               spmv_smem_bytes<VT, 2, true>(), stream, a);
          break;
        case 3:
          e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 3, true>(), g, kSpmvThreads,
                               spmv_smem_bytes<VT, 3, true>(), stream, a);
          break;
        case 4:
          e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 4, true>(), g, kSpmvThreads,
                               spmv_smem_bytes<VT, 4, true>(), stream, a);
          break;
        default:
          e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 0, true>(), g, kSpmvThreads,
                               spmv_smem_bytes<VT, 0, true>(), stream, a);
          break;
      }
      return e;
    }
  }
  switch (v) {
    case 1:
      e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 1>(), g, kSpmvThreads,
                           spmv_smem_bytes<VT, 1>(), stream, a);
      break;
    case 2:
      e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 2>(), g, kSpmvThreads,
                           spmv_smem_bytes<VT, 2>(), stream, a);
      break;
    case 3:
      e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 3>(), g, kSpmvThreads,
                           spmv_smem_bytes<VT, 3>(), stream, a);
      break;
    case 4:
      e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 4>(), g, kSpmvThreads,
                           spmv_smem_bytes<VT, 4>(), stream, a);
      break;
    default:
      e = launch_dependent(spmv_kernel_ptr<VT, M0, M1, 0>(), g, kSpmvThreads,
                           spmv_smem_bytes<VT, 0>(), stream, a);
      break;
  }
  return e;
}

#define MLSH_INST_SPMV(VT, A, B)                                                 \
  template cudaError_t launch_spmv_t<VT, A, B>(                                  \
      const CsrPlan &, const Handle &, double, const VT *, double, const VT *,   \
      VT *, const VT *, const VT *, double *, const int *, cudaStream_t);
MLSH_INST_SPMV(double, kDotNone, kDotNone)
MLSH_INST_SPMV(double, kDotW, kDotNone)
MLSH_INST_SPMV(double, kDotW, kDotSelf)
MLSH_INST_SPMV(double, kDotSelf, kDotNone)
MLSH_INST_SPMV(float, kDotNone, kDotNone)
MLSH_INST_SPMV(float, kDotW, kDotNone)
MLSH_INST_SPMV(float, kDotW, kDotSelf)
MLSH_INST_SPMV(float, kDotSelf, kDotNone)
#undef MLSH_INST_SPMV

// ------------------------------------------------------------ diag ------
template <typename VT>
__global__ void diag_kernel(int n, const int *rp, const int *ci, const VT *v,
                            VT *out, int invert) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  VT d = VT(0);
  for (int j = rp[i]; j < rp[i + 1]; ++j)
    if (ci[j] == i) d = v[j];
  out[i] = invert ? VT(1) / d : d;
}

int plan_diag(const CsrPlan &p, void *out, bool invert, cudaStream_t stream) {
  const int n = std::min(p.n_rows, p.n_cols);
  if (n <= 0) return MLSH_SUCCESS;
  const int blocks = (n + 255) / 256;
  if (p.dtype == MLSH_F64)
    diag_kernel<double><<<blocks, 256, 0, stream>>>(
        n, p.row_ptr, p.col_ind, static_cast<const double *>(p.val),
        static_cast<double *>(out), invert ? 1 : 0);
  else
    diag_kernel<float><<<blocks, 256, 0, stream>>>(
        n, p.row_ptr, p.col_ind, static_cast<const float *>(p.val),
        static_cast<float *>(out), invert ? 1 : 0);
  MLSH_CUDA_TRY(cudaGetLastError());
  return MLSH_SUCCESS;
}

int plan_inv_diag(CsrPlan &p, cudaStream_t stream, const void **out) {
  if (!p.inv_diag) {
    MLSH_CUDA_TRY(
        pool_alloc(&p.inv_diag, (size_t)std::max(p.n_rows, 1) * dtype_size(p.dtype), stream));
    p.inv_diag_valid = false;
  }
  if (!p.inv_diag_valid) {
    int st = plan_diag(p, p.inv_diag, true, stream);
    if (st != MLSH_SUCCESS) return st;
    p.inv_diag_valid = true;
  }
  *out = p.inv_diag;
  return MLSH_SUCCESS;
}

template <int NR, bool FIN, typename Body>
static int run_vec(const Handle &h, int64_t n, const Body &b) {
  RedArgs ra{h.partials, h.counters, nullptr};
  vec_kernel<NR, FIN, Body><<<vec_grid(n, h.num_sms), kVecThreads, 0, h.stream>>>(n, b, ra);
  MLSH_CUDA_TRY(cudaGetLastError());
  return MLSH_SUCCESS;
}

}  // namespace mlsh

using namespace mlsh;

// ===================================================================== C ABI
extern "C" {

int mlsh_version(void) { return 100; }

const char *mlsh_status_string(int s) {
  switch (s) {
    case MLSH_SUCCESS: return "success";
    case MLSH_SOLVER_SIZE_ERROR: return "size error";
    case MLSH_SOLVER_MAXITER: return "maxiter reached";
    case MLSH_SOLVER_BREAKDOWN: return "breakdown";
    case MLSH_SOLVER_RESIDUAL_NAN: return "residual is NaN";
    case MLSH_NOT_IMPL: return "not implemented";
    case MLSH_ERR_CUDA: return "CUDA error";
    case MLSH_ERR_INVALID_ARG: return "invalid argument";
    case MLSH_ERR_INVALID_CSR: return "invalid CRS structure";
    case MLSH_ERR_OOM: return "out of device memory";
    case MLSH_ERR_TIMEOUT: return "device wait timed out";
    case MLSH_ERR_NO_DEVICE: return "no usable CUDA device";
    default: return "unknown status";
  }
}

const char *mlsh_last_error(void) { return g_last_error; }

int mlsh_create(mlsh_handle *out) {
  if (!out) return MLSH_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MLSH_ERR_NO_DEVICE;
  auto *hs = new (std::nothrow) mlsh_handle_s();
  if (!hs) return MLSH_ERR_OOM;
  Handle &h = hs->h;
  cudaGetDevice(&h.device);
  cudaDeviceGetAttribute(&h.num_sms, cudaDevAttrMultiProcessorCount, h.device);
  int st = init_kernel_attributes();
  if (st != MLSH_SUCCESS) { delete hs; return st; }
  bool ok = cudaMalloc(&h.partials, sizeof(double) * kMaxPartialBlocks * kMaxRed) == cudaSuccess &&
            cudaMalloc(&h.counters, sizeof(unsigned) * 8) == cudaSuccess &&
            cudaMalloc(&h.scalars, sizeof(double) * 8) == cudaSuccess &&
            cudaMalloc(&h.state, sizeof(SolverState)) == cudaSuccess &&
            cudaMalloc(&h.err_flag, sizeof(int)) == cudaSuccess &&
            cudaMallocHost(&h.host_state, sizeof(SolverState)) == cudaSuccess &&
            cudaMallocHost(&h.host_scalars, sizeof(double) * 8) == cudaSuccess &&
            cudaMallocHost(&h.host_cluster, 512) == cudaSuccess &&
            cudaStreamCreateWithFlags(&h.capture_stream, cudaStreamNonBlocking) == cudaSuccess;
  if (ok) {
    ok = cudaMemset(h.counters, 0, sizeof(unsigned) * 8) == cudaSuccess &&
         cudaMemset(h.err_flag, 0, sizeof(int)) == cudaSuccess &&
         cudaMemset(h.state, 0, sizeof(SolverState)) == cudaSuccess &&
         cudaDeviceSynchronize() == cudaSuccess;
  }
  if (!ok) {
    mlsh_destroy(hs);
    return MLSH_ERR_OOM;
  }
  *out = hs;
  return MLSH_SUCCESS;
}

int mlsh_destroy(mlsh_handle hs) {
  if (!hs) return MLSH_ERR_INVALID_ARG;
  Handle &h = hs->h;
  if (h.stream) cudaStreamSynchronize(h.stream);
  release_solver_graphs(h);
  cudaFree(h.partials);
  cudaFree(h.counters);
  cudaFree(h.scalars);
  cudaFree(h.state);
  cudaFree(h.err_flag);
  cudaFreeHost(h.host_state);
  cudaFreeHost(h.host_scalars);
  cudaFreeHost(h.host_cluster);
  if (h.capture_stream) cudaStreamDestroy(h.capture_stream);
  delete hs;
  return MLSH_SUCCESS;
}

int mlsh_set_stream(mlsh_handle hs, void *stream) {
  if (!hs) return MLSH_ERR_INVALID_ARG;
  hs->h.stream = static_cast<cudaStream_t>(stream);
  return MLSH_SUCCESS;
}

int mlsh_get_stream(mlsh_handle hs, void **stream) {
  if (!hs || !stream) return MLSH_ERR_INVALID_ARG;
  *stream = hs->h.stream;
  return MLSH_SUCCESS;
}

int mlsh_synchronize(mlsh_handle hs) {
  if (!hs) return MLSH_ERR_INVALID_ARG;
  MLSH_CUDA_TRY(cudaStreamSynchronize(hs->h.stream));
  int err = 0;
  MLSH_CUDA_TRY(cudaMemcpy(&err, hs->h.err_flag, sizeof(int), cudaMemcpyDeviceToHost));
  return err != 0 ? err : MLSH_SUCCESS;
}

// --------------------------------------------------------- device memory --
int mlsh_device_alloc(size_t bytes, void **d_ptr) {
  if (!d_ptr) return MLSH_ERR_INVALID_ARG;
  *d_ptr = nullptr;
  if (bytes == 0) return MLSH_SUCCESS;
  const cudaError_t e = cudaMalloc(d_ptr, bytes);
  if (e != cudaSuccess) {
    set_last_error("cudaMalloc", e);
    cudaGetLastError();
    *d_ptr = nullptr;
    return e == cudaErrorMemoryAllocation ? MLSH_ERR_OOM : MLSH_ERR_CUDA;
  }
  return MLSH_SUCCESS;
}

int mlsh_device_free(void *d_ptr) {
  if (d_ptr) MLSH_CUDA_TRY(cudaFree(d_ptr));
  return MLSH_SUCCESS;
}

int mlsh_memcpy_h2d(mlsh_handle hs, void *d, const void *h, size_t bytes) {
  if (!hs || ((!d || !h) && bytes)) return MLSH_ERR_INVALID_ARG;
  if (!bytes) return MLSH_SUCCESS;
  MLSH_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, hs->h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(hs->h.stream));
  return MLSH_SUCCESS;
}

int mlsh_memcpy_d2h(mlsh_handle hs, void *h, const void *d, size_t bytes) {
  if (!hs || ((!d || !h) && bytes)) return MLSH_ERR_INVALID_ARG;
  if (!bytes) return MLSH_SUCCESS;
  MLSH_CUDA_TRY(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, hs->h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(hs->h.stream));
  return MLSH_SUCCESS;
}

int mlsh_memcpy_h2d_async(mlsh_handle hs, void *d, const void *h, size_t bytes) {
  if (!hs || ((!d || !h) && bytes)) return MLSH_ERR_INVALID_ARG;
  if (!bytes) return MLSH_SUCCESS;
  MLSH_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, hs->h.stream));
  return MLSH_SUCCESS;
}

int mlsh_memcpy_d2h_async(mlsh_handle hs, void *h, const void *d, size_t bytes) {
  if (!hs || ((!d || !h) && bytes)) return MLSH_ERR_INVALID_ARG;
  if (!bytes) return MLSH_SUCCESS;
  MLSH_CUDA_TRY(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, hs->h.stream));
  return MLSH_SUCCESS;
}

int mlsh_memcpy_d2d(mlsh_handle hs, void *dst, const void *src, size_t bytes) {
  if (!hs || ((!dst || !src) && bytes)) return MLSH_ERR_INVALID_ARG;
  if (!bytes) return MLSH_SUCCESS;
  MLSH_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, hs->h.stream));
  return MLSH_SUCCESS;
}

// ------------------------------------------------------------------ plan --
int mlsh_csr_plan_create(mlsh_handle hs, int n_rows, int n_cols, int nnz,
                         const int *d_row_ptr, const int *d_col_ind,
                         const void *d_val, int dtype, const int *host_row_ptr,
                         int validate, mlsh_csr_plan *out) {
  if (!hs || !out) return MLSH_ERR_INVALID_ARG;
  *out = nullptr;
  if (n_rows < 0 || n_cols < 0 || nnz < 0 || dtype_size(dtype) == 0)
    return MLSH_ERR_INVALID_ARG;
  if (n_rows > 0 && !d_row_ptr) return MLSH_ERR_INVALID_ARG;
  if (nnz > 0 && (!d_col_ind || !d_val)) return MLSH_ERR_INVALID_ARG;
  if (((uintptr_t)d_val % dtype_size(dtype)) != 0 || ((uintptr_t)d_col_ind % 4) != 0 ||
      ((uintptr_t)d_row_ptr % 4) != 0)
    return MLSH_ERR_INVALID_ARG;
  Handle &h = hs->h;
  std::vector<int> rp_copy;
  const int *rp = host_row_ptr;
  if (!rp) {
    rp_copy.resize((size_t)n_rows + 1, 0);
    if (n_rows > 0 || d_row_ptr)
      MLSH_CUDA_TRY(cudaMemcpy(rp_copy.data(), d_row_ptr, sizeof(int) * ((size_t)n_rows + 1),
                               cudaMemcpyDeviceToHost));
    rp = rp_copy.data();
  }
  if (rp[0] != 0 || rp[n_rows] != nnz) return MLSH_ERR_INVALID_CSR;
  for (int i = 0; i < n_rows; ++i)
    if (rp[i + 1] < rp[i]) return MLSH_ERR_INVALID_CSR;
  if (validate && nnz > 0) {
    std::vector<int> ci((size_t)nnz);
    MLSH_CUDA_TRY(cudaMemcpy(ci.data(), d_col_ind, sizeof(int) * (size_t)nnz,
                             cudaMemcpyDeviceToHost));
    for (int i = 0; i < nnz; ++i)
      if (ci[i] < 0 || ci[i] >= n_cols) return MLSH_ERR_INVALID_CSR;
  }
  auto *ps = new (std::nothrow) mlsh_csr_plan_s();
  if (!ps) return MLSH_ERR_OOM;
  CsrPlan &p = ps->p;
  p.handle = &h;
  p.n_rows = n_rows;
  p.n_cols = n_cols;
  p.nnz = nnz;
  p.dtype = dtype;
  p.row_ptr = d_row_ptr;
  p.col_ind = d_col_ind;
  p.val = d_val;
  std::vector<Tile> tiles;
  std::vector<LongRow> longs;
  build_tiles(rp, n_rows, tiles, longs, p.n_chunks);
  for (int i = 0; i < n_rows; ++i) p.longest_row = std::max(p.longest_row, rp[i + 1] - rp[i]);
  p.n_tiles = (int)tiles.size();
  p.n_long = (int)longs.size();
  bool ok = true;
  cudaStream_t s = h.stream;
  if (p.n_tiles > 0)
    ok = ok && pool_alloc(&p.tiles, sizeof(Tile) * tiles.size(), s) == cudaSuccess &&
         cudaMemcpyAsync(p.tiles, tiles.data(), sizeof(Tile) * tiles.size(),
                         cudaMemcpyHostToDevice, s) == cudaSuccess;
  if (p.n_long > 0)
    ok = ok && pool_alloc(&p.longs, sizeof(LongRow) * longs.size(), s) == cudaSuccess &&
         cudaMemcpyAsync(p.longs, longs.data(), sizeof(LongRow) * longs.size(),
                         cudaMemcpyHostToDevice, s) == cudaSuccess &&
         pool_alloc(&p.chunk_part, sizeof(double) * p.n_chunks, s) == cudaSuccess &&
         pool_alloc(&p.long_cnt, sizeof(unsigned) * p.n_long, s) == cudaSuccess &&
         cudaMemsetAsync(p.long_cnt, 0, sizeof(unsigned) * p.n_long, s) == cudaSuccess &&
         pool_alloc(&p.long_dot, sizeof(double) * 2 * p.n_long, s) == cudaSuccess &&
         cudaMemsetAsync(p.long_dot, 0, sizeof(double) * 2 * p.n_long, s) == cudaSuccess;
  // the plan may be used on any stream from here on
  ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
  if (!ok) {
    mlsh_csr_plan_destroy(ps);
    return MLSH_ERR_OOM;
  }
  if (dtype == MLSH_F64)
    spmv_grids<double>(p.n_tiles, h.num_sms, p.spmv_grid);
  else
    spmv_grids<float>(p.n_tiles, h.num_sms, p.spmv_grid);
  p.variant = kDefaultSpmvVariant;
  *out = ps;
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_destroy(mlsh_csr_plan ps) {
  if (!ps) return MLSH_ERR_INVALID_ARG;
  CsrPlan &p = ps->p;
  cudaStream_t s = p.handle ? p.handle->stream : nullptr;
  if (p.handle) cudaStreamSynchronize(s);
  release_plan_extras(p);
  slots_release(p);
  for (void *d : {(void *)p.tiles, (void *)p.longs, (void *)p.chunk_part, (void *)p.long_cnt,
                  (void *)p.long_dot, p.inv_diag, (void *)p.col16, (void *)p.tile_base})
    pool_free(d, s);
  if (p.handle) cudaStreamSynchronize(s);
  delete ps;
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_values_changed(mlsh_csr_plan ps) {
  if (!ps) return MLSH_ERR_INVALID_ARG;
  ps->p.inv_diag_valid = false;
  invalidate_plan_extras(ps->p);
  slots_release(ps->p);
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_info(mlsh_csr_plan ps, int *n_tiles, int *n_long_rows,
                       int64_t *spmv_bytes) {
  if (!ps) return MLSH_ERR_INVALID_ARG;
  const CsrPlan &p = ps->p;
  if (n_tiles) *n_tiles = p.n_tiles;
  if (n_long_rows) *n_long_rows = p.n_long;
  if (spmv_bytes) {
    const int64_t V = dtype_size(p.dtype);
    *spmv_bytes = (int64_t)p.nnz * (V + 4) + ((int64_t)p.n_rows + 1) * 4 +
                  (int64_t)p.n_cols * V + (int64_t)p.n_rows * V;
  }
  return MLSH_SUCCESS;
}

int mlsh_spmv(mlsh_handle hs, mlsh_csr_plan ps, double alpha, const void *d_x,
              double beta, void *d_y) {
  if (!hs || !ps) return MLSH_ERR_INVALID_ARG;
  const CsrPlan &p = ps->p;
  if (p.n_rows == 0) return MLSH_SUCCESS;
  if (!d_y || (p.n_cols > 0 && !d_x)) return MLSH_ERR_INVALID_ARG;
  const Handle &h = hs->h;
  cudaError_t e;
  if (p.dtype == MLSH_F64)
    e = launch_spmv_t<double, kDotNone, kDotNone>(
        p, h, alpha, static_cast<const double *>(d_x), beta, static_cast<const double *>(d_y),
        static_cast<double *>(d_y), nullptr, nullptr, nullptr, nullptr, h.stream);
  else
    e = launch_spmv_t<float, kDotNone, kDotNone>(
        p, h, alpha, static_cast<const float *>(d_x), beta, static_cast<const float *>(d_y),
        static_cast<float *>(d_y), nullptr, nullptr, nullptr, nullptr, h.stream);
  if (e != cudaSuccess) {
    set_last_error("spmv launch", e);
    return MLSH_ERR_CUDA;
  }
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_set_variant(mlsh_csr_plan ps, int variant) {
  if (!ps || variant < 0 || variant >= kNumSpmvVariants) return MLSH_ERR_INVALID_ARG;
  ps->p.variant = variant;
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_get_variant(mlsh_csr_plan ps, int *variant, int *n_variants) {
  if (!ps) return MLSH_ERR_INVALID_ARG;
  if (variant) *variant = ps->p.variant;
  if (n_variants) *n_variants = kNumSpmvVariants;
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_autotune(mlsh_handle hs, mlsh_csr_plan ps, const void *d_x, void *d_y,
                           int *chosen, double *best_seconds) {
  if (!hs || !ps || (ps->p.n_rows > 0 && (!d_x || !d_y))) return MLSH_ERR_INVALID_ARG;
  CsrPlan &p = ps->p;
  const Handle &h = hs->h;
  if (p.n_tiles == 0) {
    if (chosen) *chosen = p.variant;
    if (best_seconds) *best_seconds = 0.0;
    return MLSH_SUCCESS;
  }
  cudaEvent_t e0, e1;
  MLSH_CUDA_TRY(cudaEventCreate(&e0));
  MLSH_CUDA_TRY(cudaEventCreate(&e1));
  const int keep = p.variant, keep_short = p.short_max;
  int best = keep, best_short = keep_short;
  float best_ms = 1e30f;
  int st = MLSH_SUCCESS;
  // the short-row limits worth timing: 8, and 16 / 32 when some row is
  // longer than the one before (else they launch the same work)
  int limits[3] = {kShortRow, 2 * kShortRow, kMaxShortRow};
  int n_limits = p.longest_row > kShortRow ? (p.longest_row > 2 * kShortRow ? 3 : 2) : 1;
  for (int li = 0; li < n_limits && st == MLSH_SUCCESS; ++li) {
    p.short_max = limits[li];
    for (int v = 0; v < kNumSpmvVariants && st == MLSH_SUCCESS; ++v) {
      p.variant = v;
      // warm up, then time enough launches for ~1 ms of work (at least 3)
      int reps = 3;
      for (int pass = 0; pass < 2 && st == MLSH_SUCCESS; ++pass) {
        cudaEventRecord(e0, h.stream);
        for (int r = 0; r < reps; ++r) {
          st = mlsh_spmv(hs, ps, 1.0, d_x, 0.0, d_y);
          if (st != MLSH_SUCCESS) break;
        }
        cudaEventRecord(e1, h.stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (pass == 0) {
          const float per = ms / reps;
          reps = per > 0.f ? (int)std::min(200.f, std::max(3.f, 1.0f / per)) : 3;
        } else if (ms / reps < best_ms) {
          best_ms = ms / reps;
          best = v;
          best_short = limits[li];
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  p.variant = st == MLSH_SUCCESS ? best : keep;
  p.short_max = st == MLSH_SUCCESS ? best_short : keep_short;
  if (chosen) *chosen = p.variant;
  if (best_seconds) *best_seconds = best_ms * 1e-3;
  return st;
}

int mlsh_csr_plan_set_short_rows(mlsh_csr_plan ps, int max_len) {
  if (!ps || (max_len != kShortRow && max_len != 2 * kShortRow && max_len != kMaxShortRow))
    return MLSH_ERR_INVALID_ARG;
  ps->p.short_max = max_len;
  return MLSH_SUCCESS;
}

int mlsh_csr_plan_tuning(mlsh_csr_plan ps, int *variant, int *short_max) {
  if (!ps) return MLSH_ERR_INVALID_ARG;
  if (variant) *variant = ps->p.variant;
  if (short_max) *short_max = ps->p.short_max;
  return MLSH_SUCCESS;
}

int mlsh_csr_diag(mlsh_handle hs, mlsh_csr_plan ps, void *d_diag) {
  if (!hs || !ps || !d_diag) return MLSH_ERR_INVALID_ARG;
  return plan_diag(ps->p, d_diag, false, hs->h.stream);
}

// ---------------------------------------------------------- vector BLAS --
#define MLSH_VEC_CHECK(hs, dtype, n)                                   \
  if (!(hs) || dtype_size(dtype) == 0 || (n) < 0) return MLSH_ERR_INVALID_ARG; \
  if ((n) == 0) return MLSH_SUCCESS;

int mlsh_dot_device(mlsh_handle hs, int dtype, int64_t n, const void *x,
                    const void *y, double *d_result) {
  if (!hs || dtype_size(dtype) == 0 || n < 0 || !d_result) return MLSH_ERR_INVALID_ARG;
  const Handle &h = hs->h;
  if (n == 0) {
    MLSH_CUDA_TRY(cudaMemsetAsync(d_result, 0, sizeof(double), h.stream));
    return MLSH_SUCCESS;
  }
  if (dtype == MLSH_F64) {
    DotBody<double> b;
    b.x = (const double *)x; b.y = (const double *)y; b.out = d_result;
    return run_vec<1, true>(h, n, b);
  }
  DotBody<float> b;
  b.x = (const float *)x; b.y = (const float *)y; b.out = d_result;
  return run_vec<1, true>(h, n, b);
}

int mlsh_nrm2_device(mlsh_handle hs, int dtype, int64_t n, const void *x,
                     double *d_result) {
  if (!hs || dtype_size(dtype) == 0 || n < 0 || !d_result) return MLSH_ERR_INVALID_ARG;
  const Handle &h = hs->h;
  if (n == 0) {
    MLSH_CUDA_TRY(cudaMemsetAsync(d_result, 0, sizeof(double), h.stream));
    return MLSH_SUCCESS;
  }
  if (dtype == MLSH_F64) {
    Nrm2Body<double> b;
    b.x = (const double *)x; b.out = d_result;
    return run_vec<1, true>(h, n, b);
  }
  Nrm2Body<float> b;
  b.x = (const float *)x; b.out = d_result;
  return run_vec<1, true>(h, n, b);
}

static int read_scalar(const Handle &h, double *host_result) {
  MLSH_CUDA_TRY(cudaMemcpyAsync(h.host_scalars, h.scalars, sizeof(double),
                                cudaMemcpyDeviceToHost, h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  *host_result = h.host_scalars[0];
  return MLSH_SUCCESS;
}

int mlsh_dot(mlsh_handle hs, int dtype, int64_t n, const void *x, const void *y,
             double *host_result) {
  if (!host_result) return MLSH_ERR_INVALID_ARG;
  int st = mlsh_dot_device(hs, dtype, n, x, y, hs ? hs->h.scalars : nullptr);
  if (st != MLSH_SUCCESS) return st;
  return read_scalar(hs->h, host_result);
}

int mlsh_nrm2(mlsh_handle hs, int dtype, int64_t n, const void *x,
              double *host_result) {
  if (!host_result) return MLSH_ERR_INVALID_ARG;
  int st = mlsh_nrm2_device(hs, dtype, n, x, hs ? hs->h.scalars : nullptr);
  if (st != MLSH_SUCCESS) return st;
  return read_scalar(hs->h, host_result);
}

#define MLSH_ELEMENTWISE(NAME, BODY, ...)                                  \
  if (dtype == MLSH_F64) {                                                 \
    using T = double;                                                      \
    BODY<T> b;                                                             \
    __VA_ARGS__;                                                           \
    return run_vec<0, false>(hs->h, n, b);                                 \
  } else {                                                                 \
    using T = float;                                                       \
    BODY<T> b;                                                             \
    __VA_ARGS__;                                                           \
    return run_vec<0, false>(hs->h, n, b);                                 \
  }

int mlsh_axpy(mlsh_handle hs, int dtype, int64_t n, double alpha, const void *x,
              void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(axpy, AxpyBody, b.alpha = (T)alpha; b.x = (const T *)x; b.y = (T *)y)
}

int mlsh_xpay(mlsh_handle hs, int dtype, int64_t n, double alpha, const void *x,
              void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(xpay, XpayBody, b.alpha = (T)alpha; b.x = (const T *)x; b.y = (T *)y)
}

int mlsh_axpyz(mlsh_handle hs, int dtype, int64_t n, double alpha, const void *x,
               const void *y, void *z) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(axpyz, AxpyzBody, b.alpha = (T)alpha; b.x = (const T *)x;
                   b.y = (const T *)y; b.z = (T *)z)
}

int mlsh_copy(mlsh_handle hs, int dtype, int64_t n, const void *x, void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(copy, CopyBody, b.x = (const T *)x; b.y = (T *)y)
}

int mlsh_vsub(mlsh_handle hs, int dtype, int64_t n, const void *a, const void *bb,
              void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(sub, SubBody, b.a = (const T *)a; b.b = (const T *)bb; b.y = (T *)y)
}

int mlsh_vmul(mlsh_handle hs, int dtype, int64_t n, const void *a, const void *bb,
              void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(mul, MulBody, b.a = (const T *)a; b.b = (const T *)bb; b.y = (T *)y)
}

int mlsh_vreciprocal(mlsh_handle hs, int dtype, int64_t n, const void *a, void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(recip, RecipBody, b.a = (const T *)a; b.y = (T *)y)
}

int mlsh_fill(mlsh_handle hs, int dtype, int64_t n, double value, void *y) {
  MLSH_VEC_CHECK(hs, dtype, n)
  MLSH_ELEMENTWISE(fill, FillBody, b.value = (T)value; b.y = (T *)y)
}

}  // extern "C"
