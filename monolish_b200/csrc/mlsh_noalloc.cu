// mlsh_dot_noalloc: the device dot product for callers that cannot
// allocate device memory.
//
// Who needs it: a host program whose device memory is owned by a framework
// that hands out buffers from its own fixed pool and forbids other
// allocations; a latency-critical loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree may imply; a plugin that must leave the
// process's allocation state untouched.  Those callers cannot create an
// mlsh_handle (it allocates its reduction scratch with cudaMalloc).
//
// What it does: the same reduction as mlsh_dot_device (same grid, block
// size, element-to-thread mapping and fixed summation order, so the same
// result), but its scratch -- one arrival counter plus one partial sum per
// CTA -- lives in the file-scope array below, which the library's module
// places in device memory when it loads.  Every GPU that loads the library
// holds those 16,640 bytes until the process exits.
//
// Set-up: the first call on each device looks up the array's device
// address with cudaGetSymbolAddress, with that device current, and caches
// it.  That first call should therefore come before any stream capture.
// Host code never hands the array's name to a kernel: on the host that name
// is only a stand-in, not a device address.
//
// Sharing: every call uses the same array and leaves its contents behind.
// A completed launch leaves the arrival counter at zero (the last CTA resets
// it), but a launch that was aborted partway (an earlier error on the
// stream, a context that was torn down mid-kernel) can leave it counting, so
// each call still clears it (cudaMemsetAsync, no allocation) before its
// kernel runs.  Calls whose kernels overlap on the GPU (e.g. on
// two streams without ordering between them) race on the array and give
// wrong results: order them on one stream, or use mlsh_dot_device with one
// handle per stream.
#include <cuda_runtime.h>

#include <mutex>

#include "mlsh_internal.cuh"
#include "mlsh_reduce.cuh"
#include "mlsh_vec.cuh"

namespace mlsh {

// Partial sums for at most this many CTAs (one double each).
constexpr int kNoAllocMaxCtas = 2048;
// 256 bytes for the arrival counter (keeps the partials 256-byte aligned),
// then the partials.
constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocScratchBytes =
    kNoAllocCounterBytes + sizeof(double) * (size_t)kNoAllocMaxCtas;  // 16,640
// vec_grid caps the grid at kMaxVecBlocksPerSm CTAs per SM: 148 x 8 = 1,184
// on a B200, well inside the partials above; a device with more than 256
// SMs is rejected at call time.
static_assert(kMaxVecBlocksPerSm * 256 <= kNoAllocMaxCtas,
              "static scratch must hold the partials of a 256-SM device");

static __device__ __align__(256) unsigned char g_dot_scratch[kNoAllocScratchBytes];

void set_last_error_text(const char *text);

namespace {

constexpr int kMaxDevices = 64;

struct DeviceScratch {
  void *addr = nullptr;  // device address of g_dot_scratch on this device
  int num_sms = 0;
  bool ready = false;
};

std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];

// Once per device, with that device current.
int scratch_for_current_device(DeviceScratch *out) {
  int dev = 0;
  MLSH_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return MLSH_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceScratch &d = g_dev[dev];
  if (!d.ready) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
    if (e != cudaSuccess) {
      set_last_error("cudaGetSymbolAddress(g_dot_scratch)", e);
      return MLSH_ERR_CUDA;
    }
    int sms = 0;
    MLSH_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    d.addr = p;
    d.num_sms = sms;
    d.ready = true;
  }
  *out = d;
  return MLSH_SUCCESS;
}

// Same work split and summation order as vec_kernel<1, true, DotBody<T>>.
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    dot_noalloc_kernel(int64_t n, const T *x, const T *y, double *result, double *partials,
                       unsigned *counter) {
  __shared__ double red[kVecThreads / 32];
  __shared__ int last_flag;
  double acc[1] = {0.0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    acc[0] += (double)x[i] * (double)y[i];
  group_sum<1>(acc, red, threadIdx.x, kVecThreads, 0);
  if (publish_partials<1>(acc, partials, counter, &last_flag, threadIdx.x, kVecThreads, 0)) {
    double tot[1];
    reduce_partials<1>(tot, partials, (int)gridDim.x, nullptr, 0, 1, counter, red,
                       threadIdx.x, kVecThreads, 0);
    if (threadIdx.x == 0) *result = tot[0];
  }
}

}  // namespace
}  // namespace mlsh

using namespace mlsh;

extern "C" int mlsh_dot_noalloc(int dtype, int64_t n, const void *d_x, const void *d_y,
                                double *d_result, void *stream) {
  if (dtype_size(dtype) == 0 || n < 0 || !d_result || (n > 0 && (!d_x || !d_y)))
    return MLSH_ERR_INVALID_ARG;
  DeviceScratch s;
  const int st = scratch_for_current_device(&s);
  if (st != MLSH_SUCCESS) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    MLSH_CUDA_TRY(cudaMemsetAsync(d_result, 0, sizeof(double), cs));
    return MLSH_SUCCESS;
  }
  const int grid = vec_grid(n, s.num_sms);  // the grid mlsh_dot_device uses
  if (grid > kNoAllocMaxCtas) {
    set_last_error_text(
        "mlsh_dot_noalloc: this device needs more CTA partials than the static scratch "
        "holds (2048)");
    return MLSH_ERR_INVALID_ARG;
  }
  unsigned *counter = static_cast<unsigned *>(s.addr);
  double *partials =
      reinterpret_cast<double *>(static_cast<unsigned char *>(s.addr) + kNoAllocCounterBytes);
  MLSH_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), cs));
  if (dtype == MLSH_F64)
    dot_noalloc_kernel<double><<<grid, kVecThreads, 0, cs>>>(
        n, static_cast<const double *>(d_x), static_cast<const double *>(d_y), d_result,
        partials, counter);
  else
    dot_noalloc_kernel<float><<<grid, kVecThreads, 0, cs>>>(
        n, static_cast<const float *>(d_x), static_cast<const float *>(d_y), d_result,
        partials, counter);
  MLSH_CUDA_TRY(cudaGetLastError());
  return MLSH_SUCCESS;
}
