// Solve server: continuous batching of solve requests (include/mlsh.h:
// mlsh_server_*).
//
// Host side (this file): submit() queues a request; a scheduler thread
//   1. admits pending requests in arrival order while their device-memory
//      footprint fits the budget (a request larger than the whole budget
//      completes with MLSH_ERR_OOM), allocates their buffers from a
//      stream-ordered pool and uploads them;
//   2. publishes uploaded small plain-FP64 requests into one of two rings
//      (1-CTA clusters for n <= kServeRows, 16-CTA clusters up to 16 x
//      kServeRows) read by persistent serving kernels, launching a kernel
//      again whenever its ring has work and the previous launch has ended
//      (kernels exit on their own after an idle period);
//   3. hands large and mixed-precision requests to worker lanes, each with
//      its own handle and stream, which run the ordinary solve paths;
//   4. retires finished requests: copies x back, frees their memory (which
//      admits the next ones) and timestamps them.
// Device side (mlsh_cluster.cu, cluster_serve_kernel): clusters claim ring
// records while they run, solve them start to finish and flag completion,
// so requests that arrive while others are on the GPU start as soon as a
// cluster is free.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mlsh_cluster.cuh"
#include "mlsh_core.cuh"

namespace mlsh {

namespace {

constexpr unsigned kRingCapacity = 1024;
constexpr int kRingClasses = 2;                       // 1-CTA and 16-CTA clusters
constexpr int kRingClusterSize[kRingClasses] = {1, 16};
constexpr int kRingClusters[kRingClasses] = {32, 2};  // 64 SMs in all
constexpr double kRingIdleSeconds = 0.002;
constexpr double kServeBudgetSeconds = 60.0;
constexpr int kLane = 2;                              // path of lane requests

enum State { kPending, kUploading, kRunning, kDownloading, kDone };

struct Req {
  int64_t id = 0;
  mlsh_request r{};
  size_t footprint = 0;
  int path = 0;  // 0, 1: ring class; kLane: worker lane
  State state = kPending;
  void *dbuf = nullptr;
  int *d_rp = nullptr, *d_ci = nullptr;
  double *d_val = nullptr, *d_b = nullptr, *d_x = nullptr, *d_dinv = nullptr, *d_aux = nullptr;
  cudaEvent_t uploaded = nullptr, downloaded = nullptr;
  unsigned long long ring_pos = 0;
  mlsh_request_result res{};
};

struct Ring {
  ClusterSystem *rec = nullptr;        // mapped pinned
  unsigned long long *tail = nullptr;  // mapped pinned
  int *shutdown = nullptr;             // mapped pinned
  unsigned long long *head = nullptr;  // device
  ClusterSystem *d_rec = nullptr;      // device aliases of the mapped memory
  unsigned long long *d_tail = nullptr;
  int *d_shutdown = nullptr;
  unsigned long long published = 0;
  unsigned held = 0;          // admitted and not yet retired (bounds ring use)
  unsigned inflight = 0;      // published and not yet finished
  int failed = MLSH_SUCCESS;  // status of a failed kernel launch
  cudaStream_t stream = nullptr;
  cudaEvent_t kernel_done = nullptr;
  bool launched = false;
};

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

struct Server {
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_lane;
  std::deque<Req *> pending;
  std::vector<Req *> inflight;  // ring requests admitted and not done
  std::deque<Req *> lane_q;
  std::unordered_map<int64_t, Req *> all;
  size_t budget = 0, used = 0;
  int64_t next_id = 1;
  int64_t n_submitted = 0, n_done = 0;
  std::atomic<int64_t> ring_launches{0}, lane_solves{0};
  bool stop = false;
  int device = 0;
  cudaStream_t up = nullptr, down = nullptr;
  Ring ring[kRingClasses];
  std::thread sched;
  std::vector<std::thread> lanes;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// Device bytes a request holds while admitted (its matrix, vectors and, on
// a lane, the handle's work vectors and the mixed solver's FP32 copy).
size_t footprint_of(const mlsh_request &r, int path) {
  const size_t n = (size_t)r.n, nnz = (size_t)r.nnz;
  size_t b = align256(sizeof(int) * (n + 1)) + align256(sizeof(int) * nnz) +
             align256(sizeof(double) * nnz) + 4 * align256(sizeof(double) * n);
  if (path == kLane) {
    b += 8 * sizeof(double) * n + 64 * 1024;
    if (r.precision == 1) b += nnz * (4 + 2) + n * (8 + 4 + 4);
  }
  return b + 4096;
}

int route(const mlsh_request &r) {
  if (r.precision != 0 || r.n == 0) return kLane;
  if (r.n <= kServeRows) return 0;
  if (r.n <= kServeRows * 16) return 1;
  return kLane;
}

// Caller holds S.mu.
void finish(Server &S, Req *q, int status) {
  q->state = kDone;
  q->res.status = status;
  q->res.t_done = S.now();
  S.n_done++;
  S.cv_done.notify_all();
}

void release_memory(Server &S, Req *q, cudaStream_t s) {
  if (q->dbuf) cudaFreeAsync(q->dbuf, s);
  q->dbuf = nullptr;
  if (q->uploaded) cudaEventDestroy(q->uploaded);
  if (q->downloaded) cudaEventDestroy(q->downloaded);
  q->uploaded = q->downloaded = nullptr;
  std::lock_guard<std::mutex> lk(S.mu);
  S.used -= q->footprint;
}

// Allocate and upload one request (scheduler thread).
int admit(Server &S, Req *q) {
  const mlsh_request &r = q->r;
  const size_t n = (size_t)r.n, nnz = (size_t)r.nnz;
  const size_t o_rp = 0, o_ci = o_rp + align256(sizeof(int) * (n + 1));
  const size_t o_val = o_ci + align256(sizeof(int) * nnz);
  const size_t o_b = o_val + align256(sizeof(double) * nnz);
  const size_t o_x = o_b + align256(sizeof(double) * n);
  const size_t o_d = o_x + align256(sizeof(double) * n);
  const size_t o_a = o_d + align256(sizeof(double) * n);
  const size_t total = o_a + align256(sizeof(double) * n);
  MLSH_CUDA_TRY(cudaMallocAsync(&q->dbuf, total, S.up));
  char *base = static_cast<char *>(q->dbuf);
  q->d_rp = reinterpret_cast<int *>(base + o_rp);
  q->d_ci = reinterpret_cast<int *>(base + o_ci);
  q->d_val = reinterpret_cast<double *>(base + o_val);
  q->d_b = reinterpret_cast<double *>(base + o_b);
  q->d_x = reinterpret_cast<double *>(base + o_x);
  q->d_dinv = reinterpret_cast<double *>(base + o_d);
  q->d_aux = reinterpret_cast<double *>(base + o_a);
  MLSH_CUDA_TRY(cudaMemcpyAsync(q->d_rp, r.row_ptr, sizeof(int) * (n + 1),
                                cudaMemcpyHostToDevice, S.up));
  if (nnz) {
    MLSH_CUDA_TRY(cudaMemcpyAsync(q->d_ci, r.col_ind, sizeof(int) * nnz, cudaMemcpyHostToDevice,
                                  S.up));
    MLSH_CUDA_TRY(cudaMemcpyAsync(q->d_val, r.val, sizeof(double) * nnz, cudaMemcpyHostToDevice,
                                  S.up));
  }
  if (n) {
    MLSH_CUDA_TRY(cudaMemcpyAsync(q->d_b, r.b, sizeof(double) * n, cudaMemcpyHostToDevice, S.up));
    if (r.x0)
      MLSH_CUDA_TRY(cudaMemcpyAsync(q->d_x, r.x0, sizeof(double) * n, cudaMemcpyHostToDevice,
                                    S.up));
    else
      MLSH_CUDA_TRY(cudaMemsetAsync(q->d_x, 0, sizeof(double) * n, S.up));
  }
  MLSH_CUDA_TRY(cudaEventCreateWithFlags(&q->uploaded, cudaEventDisableTiming));
  MLSH_CUDA_TRY(cudaEventCreateWithFlags(&q->downloaded, cudaEventDisableTiming));
  MLSH_CUDA_TRY(cudaEventRecord(q->uploaded, S.up));
  return MLSH_SUCCESS;
}

void publish(Server &S, Req *q) {
  Ring &R = S.ring[q->path];
  const unsigned long long pos = R.published;
  ClusterSystem *rec = R.rec + (pos & (kRingCapacity - 1));
  ClusterSystem v{};
  v.rp = q->d_rp;
  v.ci = q->d_ci;
  v.val = q->d_val;
  v.b = q->d_b;
  v.x = q->d_x;
  v.dinv = q->d_dinv;
  v.aux = q->d_aux;
  v.n = q->r.n;
  v.flags = (q->r.kind == 1 ? kSysBiCGSTAB : 0) |
            (q->r.precond == MLSH_PRECOND_JACOBI ? kSysJacobi : 0);
  v.tol = q->r.tol;
  v.maxiter = q->r.maxiter;
  v.miniter = 0;
  v.status = kRunning;
  v.done = 0;
  std::memcpy(static_cast<void *>(rec), &v, sizeof(v));
  std::atomic_thread_fence(std::memory_order_release);
  __atomic_store_n(R.tail, pos + 1, __ATOMIC_RELEASE);
  R.published = pos + 1;
  R.inflight++;
  q->ring_pos = pos;
  q->state = kRunning;
}

// 0: the event has completed, 1: not yet, -1: error.
int event_state(cudaEvent_t e) {
  const cudaError_t r = cudaEventQuery(e);
  if (r == cudaSuccess) return 0;
  cudaGetLastError();
  return r == cudaErrorNotReady ? 1 : -1;
}

// Queue the copy of x back to the host (when `copy_x`) and the event that
// marks the request's device work complete.
void start_download(Server &S, Req *q, int status, bool copy_x) {
  q->res.status = status;
  if (copy_x && q->r.x_out && q->r.n > 0)
    cudaMemcpyAsync(q->r.x_out, q->d_x, sizeof(double) * q->r.n, cudaMemcpyDeviceToHost, S.down);
  cudaEventRecord(q->downloaded, S.down);
  q->state = kDownloading;
}

// Make sure the ring's kernel runs while it has unfinished records.  A
// launch that fails marks the ring failed: its head is moved past every
// published record and its requests complete with the launch's status.
void ensure_kernel(Server &S, int k) {
  Ring &R = S.ring[k];
  if (R.inflight == 0 || R.failed != MLSH_SUCCESS) return;
  if (R.launched && event_state(R.kernel_done) == 1) return;
  ServeRing sr;
  sr.rec = R.d_rec;
  sr.tail = R.d_tail;
  sr.head = R.head;
  sr.shutdown = R.d_shutdown;
  sr.capacity = kRingCapacity;
  sr.idle_ns = (unsigned long long)(kRingIdleSeconds * 1e9);
  int st = cluster_serve_launch(sr, kRingClusterSize[k], kRingClusters[k], kServeBudgetSeconds,
                                R.stream);
  if (st == MLSH_SUCCESS && cudaEventRecord(R.kernel_done, R.stream) != cudaSuccess)
    st = MLSH_ERR_CUDA;
  if (st == MLSH_SUCCESS) {
    R.launched = true;
    S.ring_launches++;
    return;
  }
  cudaGetLastError();
  R.failed = st;
  const unsigned long long head = R.published;
  cudaMemcpyAsync(R.head, &head, sizeof(head), cudaMemcpyHostToDevice, R.stream);
  cudaStreamSynchronize(R.stream);
}

void scheduler(Server *Sp) {
  Server &S = *Sp;
  cudaSetDevice(S.device);
  while (true) {
    bool progress = false;
    std::vector<Req *> to_admit;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      if (S.stop) break;
      while (!S.pending.empty()) {
        Req *q = S.pending.front();
        if (q->footprint > S.budget) {  // can never fit
          S.pending.pop_front();
          finish(S, q, MLSH_ERR_OOM);
          progress = true;
          continue;
        }
        if (S.used + q->footprint > S.budget) break;
        if (q->path != kLane && S.ring[q->path].held >= kRingCapacity) break;
        S.pending.pop_front();
        S.used += q->footprint;
        if (q->path != kLane) S.ring[q->path].held++;
        q->res.t_admit = S.now();
        to_admit.push_back(q);
      }
    }
    for (Req *q : to_admit) {
      progress = true;
      const int st = admit(S, q);
      std::lock_guard<std::mutex> lk(S.mu);
      if (st != MLSH_SUCCESS) {
        S.used -= q->footprint;
        if (q->path != kLane) S.ring[q->path].held--;
        finish(S, q, st);
        continue;
      }
      if (q->path == kLane) {
        q->state = kRunning;
        S.lane_q.push_back(q);
        S.cv_lane.notify_one();
      } else {
        q->state = kUploading;
        S.inflight.push_back(q);
      }
    }
    // publish uploaded ring requests; retire finished ones
    std::vector<Req *> keep;
    for (Req *q : S.inflight) {
      Ring &R = S.ring[q->path];
      if (q->state == kUploading) {
        const int ev = event_state(q->uploaded);
        if (ev == 0 && R.failed == MLSH_SUCCESS) {
          publish(S, q);
          progress = true;
        } else if (ev != 1) {  // upload failed, or the ring cannot run
          start_download(S, q, ev < 0 ? MLSH_ERR_CUDA : R.failed, false);
          progress = true;
        }
      } else if (q->state == kRunning) {
        ClusterSystem *rec = R.rec + (q->ring_pos & (kRingCapacity - 1));
        if (__atomic_load_n(&rec->done, __ATOMIC_ACQUIRE) != 0) {
          q->res.iters = *reinterpret_cast<volatile long long *>(&rec->iters);
          q->res.resid = *reinterpret_cast<volatile double *>(&rec->resid);
          R.inflight--;
          start_download(S, q, *reinterpret_cast<volatile int *>(&rec->status), true);
          progress = true;
        } else if (R.failed != MLSH_SUCCESS) {
          // no kernel will claim it (the ring's head was moved past it)
          R.inflight--;
          start_download(S, q, R.failed, false);
          progress = true;
        }
      } else if (q->state == kDownloading) {
        const int ev = event_state(q->downloaded);
        if (ev != 1) {
          const int status = ev == 0 ? q->res.status : MLSH_ERR_CUDA;
          release_memory(S, q, S.down);
          std::lock_guard<std::mutex> lk(S.mu);
          R.held--;
          finish(S, q, status);
          progress = true;
          continue;
        }
      }
      keep.push_back(q);
    }
    S.inflight.swap(keep);
    for (int k = 0; k < kRingClasses; ++k) ensure_kernel(S, k);
    if (!progress) {
      std::unique_lock<std::mutex> lk(S.mu);
      S.cv_work.wait_for(lk, std::chrono::microseconds(20));
    }
  }
}

void lane_worker(Server *Sp) {
  Server &S = *Sp;
  cudaSetDevice(S.device);
  cudaStream_t s;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  mlsh_handle h = nullptr;
  const int hst = mlsh_create(&h);
  if (hst == MLSH_SUCCESS) mlsh_set_stream(h, s);
  while (true) {
    Req *q = nullptr;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      S.cv_lane.wait(lk, [&] { return S.stop || !S.lane_q.empty(); });
      if (S.stop && S.lane_q.empty()) break;
      q = S.lane_q.front();
      S.lane_q.pop_front();
    }
    int status = hst;
    mlsh_solver_result res{};
    cudaStreamWaitEvent(s, q->uploaded, 0);
    mlsh_csr_plan plan = nullptr;
    if (status == MLSH_SUCCESS)
      status = mlsh_csr_plan_create(h, q->r.n, q->r.n, q->r.nnz, q->d_rp, q->d_ci, q->d_val,
                                    MLSH_F64, q->r.row_ptr, 0, &plan);
    if (status == MLSH_SUCCESS) {
      mlsh_solver_opts o;
      mlsh_solver_opts_default(&o);
      o.tol = q->r.tol;
      o.maxiter = q->r.maxiter;
      o.precond = q->r.precond;
      if (q->r.precision == 1)
        status = q->r.kind == 0
                     ? mlsh_cg_solve_mixed(h, plan, q->d_b, q->d_x, &o, q->r.inner_tol, &res)
                     : mlsh_bicgstab_solve_mixed(h, plan, q->d_b, q->d_x, &o, q->r.inner_tol,
                                                 &res);
      else
        status = q->r.kind == 0 ? mlsh_cg_solve(h, plan, q->d_b, q->d_x, &o, &res)
                                : mlsh_bicgstab_solve(h, plan, q->d_b, q->d_x, &o, &res);
      mlsh_csr_plan_destroy(plan);
    }
    if (q->r.x_out && q->r.n > 0)
      cudaMemcpyAsync(q->r.x_out, q->d_x, sizeof(double) * q->r.n, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && status >= MLSH_SUCCESS) status = MLSH_ERR_CUDA;
    q->res.iters = res.iters;
    q->res.resid = res.final_resid;
    S.lane_solves++;
    release_memory(S, q, s);
    cudaStreamSynchronize(s);
    std::lock_guard<std::mutex> lk(S.mu);
    finish(S, q, status);
  }
  if (h) mlsh_destroy(h);
  cudaStreamDestroy(s);
}

int ring_init(Ring &R) {
  MLSH_CUDA_TRY(cudaHostAlloc(&R.rec, sizeof(ClusterSystem) * kRingCapacity, cudaHostAllocMapped));
  MLSH_CUDA_TRY(cudaHostAlloc(&R.tail, 64, cudaHostAllocMapped));
  MLSH_CUDA_TRY(cudaHostAlloc(&R.shutdown, 64, cudaHostAllocMapped));
  std::memset(static_cast<void *>(R.rec), 0, sizeof(ClusterSystem) * kRingCapacity);
  *R.tail = 0;
  *R.shutdown = 0;
  MLSH_CUDA_TRY(cudaHostGetDevicePointer((void **)&R.d_rec, R.rec, 0));
  MLSH_CUDA_TRY(cudaHostGetDevicePointer((void **)&R.d_tail, R.tail, 0));
  MLSH_CUDA_TRY(cudaHostGetDevicePointer((void **)&R.d_shutdown, R.shutdown, 0));
  MLSH_CUDA_TRY(cudaMalloc(&R.head, 64));
  MLSH_CUDA_TRY(cudaMemset(R.head, 0, 64));
  MLSH_CUDA_TRY(cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking));
  MLSH_CUDA_TRY(cudaEventCreateWithFlags(&R.kernel_done, cudaEventDisableTiming));
  return MLSH_SUCCESS;
}

void ring_free(Ring &R) {
  if (R.shutdown) __atomic_store_n(R.shutdown, 1, __ATOMIC_RELEASE);
  if (R.stream) cudaStreamSynchronize(R.stream);
  if (R.rec) cudaFreeHost(R.rec);
  if (R.tail) cudaFreeHost(R.tail);
  if (R.shutdown) cudaFreeHost(R.shutdown);
  if (R.head) cudaFree(R.head);
  if (R.kernel_done) cudaEventDestroy(R.kernel_done);
  if (R.stream) cudaStreamDestroy(R.stream);
  R = Ring();
}

}  // namespace
}  // namespace mlsh

struct mlsh_server_s {
  mlsh::Server s;
};

using namespace mlsh;

extern "C" {

int mlsh_server_create(size_t budget, int n_lanes, mlsh_server *out) {
  if (!out || n_lanes < 1 || budget == 0) return MLSH_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return MLSH_ERR_NO_DEVICE;
  }
  auto *ss = new (std::nothrow) mlsh_server_s();
  if (!ss) return MLSH_ERR_OOM;
  Server &S = ss->s;
  S.budget = budget;
  cudaGetDevice(&S.device);
  // keep freed request memory in the pool up to the budget
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, S.device) == cudaSuccess) {
    uint64_t keep = budget;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  int st = MLSH_SUCCESS;
  if (cudaStreamCreateWithFlags(&S.up, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&S.down, cudaStreamNonBlocking) != cudaSuccess)
    st = MLSH_ERR_CUDA;
  for (int k = 0; k < kRingClasses && st == MLSH_SUCCESS; ++k) st = ring_init(S.ring[k]);
  if (st != MLSH_SUCCESS) {
    for (auto &R : S.ring) ring_free(R);
    if (S.up) cudaStreamDestroy(S.up);
    if (S.down) cudaStreamDestroy(S.down);
    delete ss;
    return st;
  }
  S.sched = std::thread(scheduler, &S);
  for (int i = 0; i < n_lanes; ++i) S.lanes.emplace_back(lane_worker, &S);
  *out = ss;
  return MLSH_SUCCESS;
}

int mlsh_server_submit(mlsh_server ss, const mlsh_request *r, int64_t *id) {
  if (!ss || !r || !id || r->n < 0 || r->nnz < 0 || (r->kind != 0 && r->kind != 1) ||
      (r->precision != 0 && r->precision != 1) || !r->row_ptr || (r->n > 0 && !r->b) ||
      (r->nnz > 0 && (!r->col_ind || !r->val)))
    return MLSH_ERR_INVALID_ARG;
  if (r->precision == 1 && !(r->inner_tol > 0.0 && r->inner_tol < 1.0))
    return MLSH_ERR_INVALID_ARG;
  Server &S = ss->s;
  Req *q = new (std::nothrow) Req();
  if (!q) return MLSH_ERR_OOM;
  q->r = *r;
  q->path = route(*r);
  q->footprint = footprint_of(*r, q->path);
  q->res.path = q->path == kLane ? 1 : 0;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    q->id = S.next_id++;
    q->res.t_submit = S.now();
    S.all[q->id] = q;
    S.pending.push_back(q);
    S.n_submitted++;
  }
  S.cv_work.notify_one();
  *id = q->id;
  return MLSH_SUCCESS;
}

int mlsh_server_poll(mlsh_server ss, int64_t id, mlsh_request_result *res) {
  if (!ss) return MLSH_ERR_INVALID_ARG;
  Server &S = ss->s;
  std::lock_guard<std::mutex> lk(S.mu);
  auto it = S.all.find(id);
  if (it == S.all.end()) return MLSH_ERR_INVALID_ARG;
  Req *q = it->second;
  if (q->state != kDone) return MLSH_PENDING;
  if (res) *res = q->res;
  S.all.erase(it);
  delete q;
  return MLSH_SUCCESS;
}

int mlsh_server_wait(mlsh_server ss, int64_t id, mlsh_request_result *res) {
  if (!ss) return MLSH_ERR_INVALID_ARG;
  Server &S = ss->s;
  std::unique_lock<std::mutex> lk(S.mu);
  // looked up again on every wake-up: another reader may have taken it
  S.cv_done.wait(lk, [&] {
    auto it = S.all.find(id);
    return it == S.all.end() || it->second->state == kDone;
  });
  auto it = S.all.find(id);
  if (it == S.all.end()) return MLSH_ERR_INVALID_ARG;
  Req *q = it->second;
  if (res) *res = q->res;
  S.all.erase(it);
  delete q;
  return MLSH_SUCCESS;
}

int mlsh_server_drain(mlsh_server ss) {
  if (!ss) return MLSH_ERR_INVALID_ARG;
  Server &S = ss->s;
  std::unique_lock<std::mutex> lk(S.mu);
  S.cv_done.wait(lk, [&] { return S.n_done == S.n_submitted; });
  return MLSH_SUCCESS;
}

double mlsh_server_now(mlsh_server ss) { return ss ? ss->s.now() : 0.0; }

int mlsh_server_stats(mlsh_server ss, int64_t *ring_launches, int64_t *lane_solves) {
  if (!ss) return MLSH_ERR_INVALID_ARG;
  if (ring_launches) *ring_launches = ss->s.ring_launches.load();
  if (lane_solves) *lane_solves = ss->s.lane_solves.load();
  return MLSH_SUCCESS;
}

int mlsh_server_destroy(mlsh_server ss) {
  if (!ss) return MLSH_ERR_INVALID_ARG;
  Server &S = ss->s;
  mlsh_server_drain(ss);
  {
    std::lock_guard<std::mutex> lk(S.mu);
    S.stop = true;
  }
  S.cv_work.notify_all();
  S.cv_lane.notify_all();
  if (S.sched.joinable()) S.sched.join();
  for (auto &t : S.lanes)
    if (t.joinable()) t.join();
  for (auto &R : S.ring) ring_free(R);
  if (S.up) cudaStreamDestroy(S.up);
  if (S.down) cudaStreamDestroy(S.down);
  for (auto &kv : S.all) delete kv.second;
  delete ss;
  return MLSH_SUCCESS;
}

}  // extern "C"
