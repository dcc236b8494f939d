// Batched solves of independent systems on the cluster engine
// (include/mlsh.h: mlsh_batch_*).
//
// Systems are grouped by the cluster size their row count needs and sorted
// largest first inside a group (longest jobs start first, which bounds the
// tail).  Each group is one persistent launch of the cluster kernel with as
// many clusters as fit the device; clusters pull systems from the group's
// queue.  Groups run on separate streams, largest cluster size first, so
// when one group's queue drains its SMs are taken by the next group's
// clusters.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "mlsh_cluster.cuh"
#include "mlsh_core.cuh"

namespace mlsh {

constexpr int kMaxBatchGroups = 128;
constexpr int kMaxRowsPerCta = 16384;  // the widest slice the engine takes
constexpr int kMinRowsPerCta = 1024;

struct BatchGroup {
  int csize = 1;
  int rpc = 1024;
  int first = 0;  // index of the group's first record in the system array
  int count = 0;
  cudaStream_t stream = nullptr;
};

struct Batch {
  Handle *handle = nullptr;
  int n_systems = 0;
  int dtype = MLSH_F64;
  int64_t total_rows = 0;
  std::vector<int64_t> row_off;
  std::vector<int> order[3];  // per kind: record i solves system order[i]
  const int *row_ptr = nullptr;
  const int *col_ind = nullptr;
  const void *val = nullptr;
  std::vector<BatchGroup> groups[3];  // per kind (CG, BiCGSTAB, mixed CG)
  float *val32 = nullptr;             // FP32 copy of the values (mixed CG)
  // rows-per-CTA cap per kind: a system takes the widest slice that fits
  // under it, which sets both its cluster shape and the group (bin) it
  // joins; mlsh_batch_autotune times the candidates
  int rpc_cap[3] = {kMaxRowsPerCta, kMaxRowsPerCta, kMaxRowsPerCta};
  ClusterSystem *d_sys = nullptr;     // n_systems records
  ClusterSystem *h_sys = nullptr;     // pinned mirror
  unsigned *d_queue = nullptr;        // one counter per group
  void *ws = nullptr;                 // inverse diagonal + BiCGSTAB r0
  cudaEvent_t done_event = nullptr;
};

namespace {

// Groups for one kind: systems by needed cluster size (largest first).
// Each system takes the widest slice (rows per CTA, a power of two up to
// B.rpc_cap[kind]) that fits the engine; when none under the cap fits, the
// narrowest that does.
int build_groups(Batch &B, int kind, std::vector<BatchGroup> &groups,
                 std::vector<int> &order) {
  const int cap = B.rpc_cap[kind];
  const int n = B.n_systems;
  const int dt = kind == 2 ? MLSH_F32 : B.dtype;  // mixed CG iterates in FP32
  std::vector<int> rpc(n), cs(n);
  for (int k = 0; k < n; ++k) {
    const int64_t nk = B.row_off[k + 1] - B.row_off[k];
    // one CTA while the system fits one; otherwise the widest slices
    int r = cluster_rows_for(kind, dt, nk, 0);
    if (r == 0) return MLSH_ERR_INVALID_ARG;
    int single = cluster_rows_for(kind, dt, nk, (int)std::max<int64_t>(nk, 1));
    if (single > 0 && nk <= single && single <= cap) {
      r = single;
    } else {
      // largest slice under the cap that fits: fewer CTAs per system
      int best = r;
      for (int t = r; t <= std::min(cap, kMaxRowsPerCta); t <<= 1) {
        const int ok = cluster_rows_for(kind, dt, nk, t);
        if (ok == t) best = t;
      }
      r = best;
    }
    rpc[k] = r;
    cs[k] = (int)((nk + r - 1) / r);
    if (cs[k] < 1) cs[k] = 1;
  }
  order.resize(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (cs[a] != cs[b]) return cs[a] > cs[b];
    if (rpc[a] != rpc[b]) return rpc[a] > rpc[b];
    const int64_t na = B.row_off[a + 1] - B.row_off[a];
    const int64_t nb = B.row_off[b + 1] - B.row_off[b];
    return na > nb;
  });
  groups.clear();
  for (int i = 0; i < n; ++i) {
    const int k = order[i];
    if (groups.empty() || groups.back().csize != cs[k] || groups.back().rpc != rpc[k]) {
      if ((int)groups.size() == kMaxBatchGroups) return MLSH_ERR_INVALID_ARG;
      BatchGroup g;
      g.csize = cs[k];
      g.rpc = rpc[k];
      g.first = i;
      g.count = 0;
      groups.push_back(g);
    }
    ++groups.back().count;
  }
  return MLSH_SUCCESS;
}

// Forget one kind's grouping (and its streams) so the next run rebuilds it.
void drop_groups(Batch &B, int kind) {
  for (BatchGroup &g : B.groups[kind])
    if (g.stream) {
      cudaStreamSynchronize(g.stream);
      cudaStreamDestroy(g.stream);
    }
  B.groups[kind].clear();
}

void free_batch(Batch &B) {
  for (auto &gl : B.groups)
    for (auto &g : gl)
      if (g.stream) cudaStreamDestroy(g.stream);
  cudaFree(B.d_sys);
  cudaFreeHost(B.h_sys);
  cudaFree(B.d_queue);
  cudaFree(B.ws);
  cudaFree(B.val32);
  if (B.done_event) cudaEventDestroy(B.done_event);
}

__global__ void values_to_f32(const double *v, int64_t n, float *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)v[i];
}

}  // namespace
}  // namespace mlsh

struct mlsh_batch_s {
  mlsh::Batch b;
};

using namespace mlsh;

extern "C" {

int mlsh_batch_create(mlsh_handle hs, int n_systems, const int64_t *row_off,
                      const int *d_row_ptr, const int *d_col_ind, const void *d_val, int dtype,
                      mlsh_batch *out) {
  if (!hs || !out || n_systems < 0 || (n_systems > 0 && !row_off) || dtype_size(dtype) == 0)
    return MLSH_ERR_INVALID_ARG;
  *out = nullptr;
  auto *bs = new (std::nothrow) mlsh_batch_s();
  if (!bs) return MLSH_ERR_OOM;
  Batch &B = bs->b;
  B.handle = &hs->h;
  B.n_systems = n_systems;
  B.dtype = dtype;
  B.row_off.assign(row_off, row_off + n_systems + 1);
  B.total_rows = n_systems > 0 ? row_off[n_systems] : 0;
  for (int k = 0; k < n_systems; ++k)
    if (row_off[k + 1] < row_off[k]) {
      delete bs;
      return MLSH_ERR_INVALID_ARG;
    }
  B.row_ptr = d_row_ptr;
  B.col_ind = d_col_ind;
  B.val = d_val;
  // CG grouping now (it also validates the sizes); BiCGSTAB on first use
  {
    const int st = build_groups(B, 0, B.groups[0], B.order[0]);
    if (st != MLSH_SUCCESS) {
      delete bs;
      return st;
    }
  }
  const size_t esz = (size_t)dtype_size(dtype);
  const size_t n_rec = (size_t)std::max(n_systems, 1);
  bool ok = cudaMalloc(&B.d_sys, sizeof(ClusterSystem) * n_rec) == cudaSuccess &&
            cudaMallocHost(&B.h_sys, sizeof(ClusterSystem) * n_rec) == cudaSuccess &&
            cudaMalloc(&B.d_queue, sizeof(unsigned) * kMaxBatchGroups) == cudaSuccess &&
            cudaMalloc(&B.ws, 2 * esz * (size_t)std::max<int64_t>(B.total_rows, 1) + 256) ==
                cudaSuccess &&
            cudaEventCreateWithFlags(&B.done_event, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_batch(B);
    delete bs;
    return MLSH_ERR_OOM;
  }
  *out = bs;
  return MLSH_SUCCESS;
}

int mlsh_batch_destroy(mlsh_batch bs) {
  if (!bs) return MLSH_ERR_INVALID_ARG;
  if (bs->b.handle) cudaStreamSynchronize(bs->b.handle->stream);
  free_batch(bs->b);
  delete bs;
  return MLSH_SUCCESS;
}

}  // extern "C"

namespace mlsh {
namespace {

// One batched solve of `kind` (0 CG, 1 BiCGSTAB, 2 mixed CG with refresh
// factor `delta`).
int batch_run(Handle &h, Batch &B, int kind, const void *d_b, void *d_x, const double *host_tol,
              const mlsh_solver_opts *opts, double delta, int *host_status,
              int64_t *host_iters, double *host_resid) {
  if (B.n_systems == 0) return MLSH_SUCCESS;
  if (!d_b || !d_x) return MLSH_ERR_INVALID_ARG;
  std::vector<BatchGroup> &groups = B.groups[kind];
  std::vector<int> &order = B.order[kind];
  if (groups.empty()) {
    const int st = build_groups(B, kind, groups, order);
    if (st != MLSH_SUCCESS) return st;
  }
  if ((int)order.size() != B.n_systems) return MLSH_ERR_INVALID_ARG;
  const int dt = kind == 2 ? MLSH_F32 : B.dtype;   // the iteration's type
  const size_t esz = (size_t)dtype_size(B.dtype);  // b, x, values
  const size_t isz = (size_t)dtype_size(dt);       // work vectors
  char *ws = static_cast<char *>(B.ws);
  const bool jac = opts->precond == MLSH_PRECOND_JACOBI;
  for (int i = 0; i < B.n_systems; ++i) {
    const int k = order[i];
    ClusterSystem &S = B.h_sys[i];
    std::memset(&S, 0, sizeof(S));
    const int64_t r0 = B.row_off[k];
    S.rp = B.row_ptr + r0;
    S.ci = B.col_ind;
    S.b = static_cast<const char *>(d_b) + r0 * esz;
    S.x = static_cast<char *>(d_x) + r0 * esz;
    S.dinv = ws + r0 * isz;
    if (kind == 2) {
      S.val = B.val32;
      S.aux = const_cast<void *>(B.val);  // the FP64 values of the true residual
    } else {
      S.val = B.val;
      S.aux = ws + (B.total_rows + r0) * isz;
    }
    S.n = (int)(B.row_off[k + 1] - r0);
    S.tol = host_tol ? host_tol[k] : opts->tol;
    S.maxiter = opts->maxiter;
    S.miniter = opts->miniter;
    S.status = kRunning;
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(B.d_sys, B.h_sys, sizeof(ClusterSystem) * B.n_systems,
                                cudaMemcpyHostToDevice, h.stream));
  MLSH_CUDA_TRY(cudaMemsetAsync(B.d_queue, 0, sizeof(unsigned) * kMaxBatchGroups, h.stream));
  MLSH_CUDA_TRY(cudaEventRecord(B.done_event, h.stream));
  // one stream per group, ordered after the uploads on the handle's stream
  const int n_groups = (int)groups.size();
  for (int gi = 0; gi < n_groups; ++gi) {
    BatchGroup &g = groups[gi];
    if (!g.stream) MLSH_CUDA_TRY(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    MLSH_CUDA_TRY(cudaStreamWaitEvent(g.stream, B.done_event, 0));
    int n_clusters = cluster_max_active(kind, dt, jac, g.rpc, g.csize);
    if (n_clusters < 1) return MLSH_NOT_IMPL;
    n_clusters = std::min(n_clusters, g.count);
    const int st = cluster_launch(h, kind, dt, jac, B.d_sys + g.first, g.count, B.d_queue + gi,
                                  g.rpc, g.csize, n_clusters, cluster_budget(opts), g.stream,
                                  delta);
    if (st != MLSH_SUCCESS) return st;
  }
  for (int gi = 0; gi < n_groups; ++gi) {
    cudaEvent_t ev;
    MLSH_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    MLSH_CUDA_TRY(cudaEventRecord(ev, groups[gi].stream));
    MLSH_CUDA_TRY(cudaStreamWaitEvent(h.stream, ev, 0));
    cudaEventDestroy(ev);
  }
  MLSH_CUDA_TRY(cudaMemcpyAsync(B.h_sys, B.d_sys, sizeof(ClusterSystem) * B.n_systems,
                                cudaMemcpyDeviceToHost, h.stream));
  MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
  int first_bad = MLSH_SUCCESS;
  for (int i = 0; i < B.n_systems; ++i) {
    const int k = order[i];
    const ClusterSystem &S = B.h_sys[i];
    if (host_status) host_status[k] = S.status;
    if (host_iters) host_iters[k] = S.iters;
    if (host_resid) host_resid[k] = S.resid;
    if (S.status != MLSH_SUCCESS && first_bad == MLSH_SUCCESS) first_bad = S.status;
  }
  return first_bad;
}

// The FP32 copy of the values the mixed-precision solves iterate with.
int ensure_val32(Handle &h, Batch &B) {
  if (B.dtype != MLSH_F64) return MLSH_ERR_INVALID_ARG;
  if (B.n_systems > 0 && !B.val32) {
    int nnz = 0;
    MLSH_CUDA_TRY(cudaMemcpy(&nnz, B.row_ptr + B.total_rows, sizeof(int),
                             cudaMemcpyDeviceToHost));
    if (cudaMalloc(&B.val32, sizeof(float) * (size_t)std::max(nnz, 1)) != cudaSuccess) {
      cudaGetLastError();
      B.val32 = nullptr;
      return MLSH_ERR_OOM;
    }
    if (nnz > 0) {
      const unsigned g = (unsigned)std::min<int64_t>(((int64_t)nnz + 255) / 256, 148 * 16);
      values_to_f32<<<g, 256, 0, h.stream>>>(static_cast<const double *>(B.val), nnz,
                                             B.val32);
      MLSH_CUDA_TRY(cudaGetLastError());
    }
  }
  return MLSH_SUCCESS;
}

}  // namespace
}  // namespace mlsh

extern "C" {

int mlsh_batch_solve(mlsh_handle hs, mlsh_batch bs, int kind, const void *d_b, void *d_x,
                     const double *host_tol, const mlsh_solver_opts *opts, int *host_status,
                     int64_t *host_iters, double *host_resid) {
  if (!hs || !bs || !opts || (kind != 0 && kind != 1)) return MLSH_ERR_INVALID_ARG;
  return batch_run(hs->h, bs->b, kind, d_b, d_x, host_tol, opts, 0.0, host_status, host_iters,
                   host_resid);
}

int mlsh_batch_autotune(mlsh_handle hs, mlsh_batch bs, int kind, const void *d_b, void *d_x,
                        const double *host_tol, const mlsh_solver_opts *opts, double inner_tol,
                        int *chosen_cap, double *best_seconds) {
  if (!hs || !bs || !opts || kind < 0 || kind > 2 || (bs->b.n_systems > 0 && (!d_b || !d_x)))
    return MLSH_ERR_INVALID_ARG;
  if (kind == 2 && !(inner_tol > 0.0 && inner_tol < 1.0)) return MLSH_ERR_INVALID_ARG;
  Batch &B = bs->b;
  Handle &h = hs->h;
  if (kind == 2) {
    const int vs = ensure_val32(h, B);
    if (vs != MLSH_SUCCESS) return vs;
  }
  const int keep = B.rpc_cap[kind];
  if (B.n_systems == 0) {
    if (chosen_cap) *chosen_cap = keep;
    if (best_seconds) *best_seconds = 0.0;
    return MLSH_SUCCESS;
  }
  // x is the initial guess: kept aside and put back before every timed solve
  const size_t xbytes = (size_t)dtype_size(B.dtype) * (size_t)B.total_rows;
  void *x0 = nullptr;
  MLSH_CUDA_TRY(cudaMalloc(&x0, xbytes));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int st = MLSH_SUCCESS;
  if (cudaMemcpyAsync(x0, d_x, xbytes, cudaMemcpyDeviceToDevice, h.stream) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    st = MLSH_ERR_CUDA;
  int best = keep, last_groups = -1;
  float best_ms = 1e30f;
  for (int cap = kMinRowsPerCta; cap <= kMaxRowsPerCta && st == MLSH_SUCCESS; cap <<= 1) {
    B.rpc_cap[kind] = cap;
    drop_groups(B, kind);
    st = build_groups(B, kind, B.groups[kind], B.order[kind]);
    if (st != MLSH_SUCCESS) break;
    // caps that leave the grouping as the previous one launch the same work
    int sig = 0;
    for (const BatchGroup &g : B.groups[kind]) sig = sig * 31 + g.rpc * 7 + g.csize;
    if (sig == last_groups) continue;
    last_groups = sig;
    if (cudaMemcpyAsync(d_x, x0, xbytes, cudaMemcpyDeviceToDevice, h.stream) != cudaSuccess ||
        cudaEventRecord(e0, h.stream) != cudaSuccess) {
      st = MLSH_ERR_CUDA;
      break;
    }
    const int rs = batch_run(h, B, kind, d_b, d_x, host_tol, opts, kind == 2 ? inner_tol : 0.0,
                             nullptr, nullptr, nullptr);
    if (rs == MLSH_NOT_IMPL) {  // a group shape the engine cannot launch
      for (const BatchGroup &g : B.groups[kind])
        if (g.stream) cudaStreamSynchronize(g.stream);  // groups launched before it
      continue;
    }
    if (rs < MLSH_NOT_IMPL) {  // a library error, not a solver status
      st = rs;
      break;
    }
    cudaEventRecord(e1, h.stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = cap;
    }
  }
  B.rpc_cap[kind] = st == MLSH_SUCCESS ? best : keep;
  drop_groups(B, kind);
  const int sg = build_groups(B, kind, B.groups[kind], B.order[kind]);
  if (st == MLSH_SUCCESS) st = sg;
  cudaMemcpyAsync(d_x, x0, xbytes, cudaMemcpyDeviceToDevice, h.stream);
  cudaStreamSynchronize(h.stream);
  cudaFree(x0);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (chosen_cap) *chosen_cap = B.rpc_cap[kind];
  if (best_seconds) *best_seconds = best_ms * 1e-3;
  return st;
}

int mlsh_batch_info(mlsh_batch bs, int kind, int *rows_per_cta_cap, int *n_groups) {
  if (!bs || kind < 0 || kind > 2) return MLSH_ERR_INVALID_ARG;
  Batch &B = bs->b;
  if (B.groups[kind].empty() && B.n_systems > 0) {
    const int st = build_groups(B, kind, B.groups[kind], B.order[kind]);
    if (st != MLSH_SUCCESS) return st;
  }
  if (rows_per_cta_cap) *rows_per_cta_cap = B.rpc_cap[kind];
  if (n_groups) *n_groups = (int)B.groups[kind].size();
  return MLSH_SUCCESS;
}

int mlsh_batch_cg_solve_mixed(mlsh_handle hs, mlsh_batch bs, const void *d_b, void *d_x,
                              const double *host_tol, const mlsh_solver_opts *opts,
                              double inner_tol, int *host_status, int64_t *host_iters,
                              double *host_resid) {
  if (!hs || !bs || !opts || !(inner_tol > 0.0) || !(inner_tol < 1.0))
    return MLSH_ERR_INVALID_ARG;
  Batch &B = bs->b;
  Handle &h = hs->h;
  const int st = ensure_val32(h, B);
  if (st != MLSH_SUCCESS) return st;
  return batch_run(h, B, 2, d_b, d_x, host_tol, opts, inner_tol, host_status, host_iters,
                   host_resid);
}

}  // extern "C"
