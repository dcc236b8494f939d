// Cluster-resident CG / BiCGSTAB kernels and their launchers (see
// mlsh_cluster.cuh for the design).
//
// The per-system solve bodies are device functions used by two kinds of
// kernel: the queue kernels (single solves and batches: clusters take the
// next system index from an atomic counter) and the serving kernel
// (clusters claim records that the host publishes into a ring while the
// kernel runs -- continuous batching; see mlsh_serve.cu).
#include <cuda_runtime.h>

#include <cuda/atomic>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "mlsh_cluster.cuh"
#include "mlsh_core.cuh"

namespace mlsh {

namespace cgs = cooperative_groups;

// Shared state of one CTA of the cluster engine.
struct ClusterShared {
  double slots[2 * kClusterMaxNR * kMaxClusterSize];  // [parity][k][rank]
  double red_warp[32 * 3];
  void *remote_vec[kMaxClusterSize];      // gathered-vector slice of each CTA
  double *remote_slots[kMaxClusterSize];
  ClusterSystem sys;                      // serving: this CTA's copy of the record
  unsigned long long sys_idx;
};

// Per-CTA view of the engine (one per kernel).
struct ClusterEnv {
  cgs::cluster_group &cl;
  ClusterShared &sh;
  unsigned char *dyn;
  unsigned csize, rank;
  int shift, rpc, mask;
  int parity;
};

struct SolveOut {
  int status;
  long long iters;
  double resid;
};

#define MLSH_FOR_OWN_ROWS(i, nloc) \
  for (int i = (int)threadIdx.x; i < (nloc); i += kClusterThreads)

template <typename T>
__device__ __forceinline__ void cluster_jacobi_setup(const int *rp, const int *ci, const T *val,
                                                     T *dinv, int row0, int nloc, bool jac) {
  if (!jac) return;
  MLSH_FOR_OWN_ROWS(i, nloc) {
    const int row = row0 + i;
    T d = T(0);
    for (int j = __ldg(rp + row); j < __ldg(rp + row + 1); ++j)
      if (__ldg(ci + j) == row) d = __ldg(val + j);
    dinv[row] = T(1) / d;
  }
}

template <int NR>
__device__ __forceinline__ void env_sum(ClusterEnv &E, double (&v)[NR]) {
  cluster_sum<NR>(v, E.sh.red_warp, E.sh.remote_slots, E.sh.slots, E.parity, E.csize, E.rank,
                  E.cl);
  E.parity ^= 1;
}

// ------------------------------------------------------------------- CG --
// src/equation/cg.cpp:13-86 on one system; dynamic smem: r, g (= p), q.
// Inlined into each kernel so that `jac` is a constant where the kernel
// fixes it.
template <typename T>
__device__ __forceinline__ SolveOut cg_system(ClusterEnv &E, const ClusterSystem &S, bool jac,
                                              unsigned long long budget_ns) {
  const int RPC = E.rpc;
  T *r = reinterpret_cast<T *>(E.dyn);
  T *g = r + RPC;
  T *q = g + RPC;
  T *const *remote = reinterpret_cast<T *const *>(E.sh.remote_vec);
  const int rank = (int)E.rank, shift = E.shift, mask = E.mask;
  const int n = S.n;
  const int row0 = rank * RPC;
  const int nloc = max(0, min(RPC, n - row0));
  const int *rp = S.rp, *ci = S.ci;
  const T *val = static_cast<const T *>(S.val);
  const T *b = static_cast<const T *>(S.b);
  T *x = static_cast<T *>(S.x);
  T *dinv = static_cast<T *>(S.dinv);
  const double tol = S.tol;
  const long long maxiter = S.maxiter, miniter = S.miniter;
  double *hist = S.hist;
  const long long hist_cap = S.hist_cap;
  const uint64_t t0 = global_timer_ns();

  cluster_jacobi_setup<T>(rp, ci, val, dinv, row0, nloc, jac);
  MLSH_FOR_OWN_ROWS(i, nloc) g[i] = x[row0 + i];
  E.cl.sync();
  // r = b - A x0 (cg.cpp:39-40), z = M r, p = z (cg.cpp:43-44)
  double s2[2] = {0.0, 0.0};
  MLSH_FOR_OWN_ROWS(i, nloc) {
    const int row = row0 + i;
    const T qv = cluster_row_dot<T>(rp, ci, val, row, g, remote, shift, mask, rank);
    const T ri = b[row] - qv;
    r[i] = ri;
    const T zi = jac ? dinv[row] * ri : ri;
    q[i] = zi;
    s2[0] += (double)zi * (double)ri;
    s2[1] += (double)ri * (double)ri;
  }
  env_sum<2>(E, s2);
  double rz = s2[0], rr = s2[1];
  MLSH_FOR_OWN_ROWS(i, nloc) g[i] = q[i];
  long long it = 0;
  int status = maxiter <= 0 ? MLSH_SOLVER_MAXITER : kRunning;
  double resid = cl_resid<T>(rr);
  E.cl.sync();

  while (status == kRunning) {
    // q = A p, (p, q)
    double pq[1] = {0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const T qv = cluster_row_dot<T>(rp, ci, val, row0 + i, g, remote, shift, mask, rank);
      q[i] = qv;
      pq[0] += (double)g[i] * (double)qv;
    }
    env_sum<1>(E, pq);
    const T alpha = (T)(rz / pq[0]);
    // x += alpha p; r -= alpha q; (z, r), (r, r); time budget
    double s3[3] = {0.0, 0.0, 0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      const T pi = g[i], qi = q[i];
      x[row] = alpha * pi + x[row];
      const T ri = -alpha * qi + r[i];
      r[i] = ri;
      const T zi = jac ? dinv[row] * ri : ri;
      s3[0] += (double)zi * (double)ri;
      s3[1] += (double)ri * (double)ri;
    }
    if (rank == 0 && threadIdx.x == 0 && global_timer_ns() - t0 > budget_ns) s3[2] = 1.0;
    env_sum<3>(E, s3);
    rr = s3[1];
    ++it;
    resid = cl_resid<T>(rr);
    if (rank == 0 && threadIdx.x == 0 && hist != nullptr && it <= hist_cap) hist[it - 1] = resid;
    if (resid < tol && miniter <= it) status = MLSH_SUCCESS;
    else if (isnan(resid)) status = MLSH_SOLVER_RESIDUAL_NAN;
    else if (it >= maxiter) status = MLSH_SOLVER_MAXITER;
    else if (s3[2] > 0.0) status = MLSH_ERR_TIMEOUT;
    if (status != kRunning) break;
    const T beta = (T)(s3[0] / rz);
    rz = s3[0];
    // p = z + beta p (cg.cpp:59)
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const T zi = jac ? dinv[row0 + i] * r[i] : r[i];
      g[i] = zi + beta * g[i];
    }
    E.cl.sync();
  }
  // every x write above precedes the last cluster barrier (inside env_sum)
  return SolveOut{status, it, resid};
}

// ------------------------------------------------------------- BiCGSTAB --
// src/equation/bicgstab.cpp:13-135 on one system; dynamic smem: r, p, v,
// s, t, g (= p-hat, then s-hat).
template <typename T>
__device__ __forceinline__ SolveOut bicgstab_system(ClusterEnv &E, const ClusterSystem &S,
                                                    bool jac, unsigned long long budget_ns) {
  const int RPC = E.rpc;
  T *r = reinterpret_cast<T *>(E.dyn);
  T *p = r + RPC;
  T *v = p + RPC;
  T *s = v + RPC;
  T *t = s + RPC;
  T *g = t + RPC;
  T *const *remote = reinterpret_cast<T *const *>(E.sh.remote_vec);
  const int rank = (int)E.rank, shift = E.shift, mask = E.mask;
  const int n = S.n;
  const int row0 = rank * RPC;
  const int nloc = max(0, min(RPC, n - row0));
  const int *rp = S.rp, *ci = S.ci;
  const T *val = static_cast<const T *>(S.val);
  const T *b = static_cast<const T *>(S.b);
  T *x = static_cast<T *>(S.x);
  T *dinv = static_cast<T *>(S.dinv);
  T *r0 = static_cast<T *>(S.aux);
  const double tol = S.tol;
  const long long maxiter = S.maxiter, miniter = S.miniter;
  double *hist = S.hist;
  const long long hist_cap = S.hist_cap;
  const uint64_t t0 = global_timer_ns();

  cluster_jacobi_setup<T>(rp, ci, val, dinv, row0, nloc, jac);
  MLSH_FOR_OWN_ROWS(i, nloc) g[i] = x[row0 + i];
  E.cl.sync();
  // r = b - A x, r0 = r (bicgstab.cpp:47-51)
  double s2[2] = {0.0, 0.0};
  MLSH_FOR_OWN_ROWS(i, nloc) {
    const int row = row0 + i;
    const T ri = b[row] - cluster_row_dot<T>(rp, ci, val, row, g, remote, shift, mask, rank);
    r[i] = ri;
    r0[row] = ri;
    s2[0] += (double)ri * (double)ri;
    s2[1] += (double)ri * (double)ri;
  }
  env_sum<2>(E, s2);
  double rho = s2[0], rr = s2[1], rho_old = 1.0, alpha_d = 1.0, omega_d = 1.0;
  long long it = 0;
  double resid = cl_resid<T>(rr);
  int status = kRunning;
  if (maxiter <= 0) {
    status = MLSH_SOLVER_MAXITER;
  } else if (rho == 0.0) {
    status = MLSH_SOLVER_BREAKDOWN;
    it = 1;
  }

  while (status == kRunning) {
    // p = r + beta (p - omega v) (bicgstab.cpp:66-74); p-hat = M p
    const T beta = (T)((rho / rho_old) * (alpha_d / omega_d));
    const T omega_t = (T)omega_d;
    MLSH_FOR_OWN_ROWS(i, nloc) {
      T pi;
      if (it == 0) {
        pi = r[i];
      } else {
        const T tmp = -omega_t * v[i] + p[i];
        pi = r[i] + beta * tmp;
      }
      p[i] = pi;
      g[i] = jac ? dinv[row0 + i] * pi : pi;
    }
    E.cl.sync();
    // v = A p-hat; alpha = rho / (v, r0)
    double vr[1] = {0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      const T vv = cluster_row_dot<T>(rp, ci, val, row, g, remote, shift, mask, rank);
      v[i] = vv;
      vr[0] += (double)vv * (double)r0[row];
    }
    env_sum<1>(E, vr);
    const T alpha = (T)(rho / vr[0]);
    alpha_d = (double)alpha;
    // s = r - alpha v; s-hat = M s
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const T si = -alpha * v[i] + r[i];
      s[i] = si;
      g[i] = jac ? dinv[row0 + i] * si : si;
    }
    E.cl.sync();
    // t = A s-hat; omega = (t, s) / (t, t)
    double tw[2] = {0.0, 0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const T tv = cluster_row_dot<T>(rp, ci, val, row0 + i, g, remote, shift, mask, rank);
      t[i] = tv;
      tw[0] += (double)tv * (double)s[i];
      tw[1] += (double)tv * (double)tv;
    }
    env_sum<2>(E, tw);
    const T omega = (T)(tw[0] / tw[1]);
    if (omega == T(0)) {  // bicgstab.cpp:93-98
      status = MLSH_SOLVER_BREAKDOWN;
      ++it;
      break;
    }
    omega_d = (double)omega;
    // x += alpha p-hat + omega s-hat; r = s - omega t; (r, r0), (r, r)
    double s3[3] = {0.0, 0.0, 0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      const T di = jac ? dinv[row] : T(1);
      const T ph = jac ? di * p[i] : p[i];
      const T shh = jac ? di * s[i] : s[i];
      T xi = alpha * ph + x[row];
      xi = omega * shh + xi;
      x[row] = xi;
      const T ri = -omega * t[i] + s[i];
      r[i] = ri;
      s3[0] += (double)ri * (double)r0[row];
      s3[1] += (double)ri * (double)ri;
    }
    if (rank == 0 && threadIdx.x == 0 && global_timer_ns() - t0 > budget_ns) s3[2] = 1.0;
    env_sum<3>(E, s3);
    rr = s3[1];
    ++it;
    resid = cl_resid<T>(rr);
    if (rank == 0 && threadIdx.x == 0 && hist != nullptr && it <= hist_cap) hist[it - 1] = resid;
    if (resid < tol && miniter <= it) status = MLSH_SUCCESS;
    else if (isnan(resid)) status = MLSH_SOLVER_RESIDUAL_NAN;
    else if (it >= maxiter) status = MLSH_SOLVER_MAXITER;
    else if (s3[2] > 0.0) status = MLSH_ERR_TIMEOUT;
    if (status != kRunning) break;
    rho_old = rho;
    rho = s3[0];
    if (rho == 0.0) {  // next iteration's breakdown check (bicgstab.cpp:58-63)
      status = MLSH_SOLVER_BREAKDOWN;
      ++it;
    }
  }
  // every x write above precedes the last cluster barrier (inside env_sum)
  return SolveOut{status, it, resid};
}

// ----------------------------------------------------------- mixed CG --
// Jacobi-CG with FP32 iteration vectors and FP32 matrix values, the
// solution and the true residual in FP64: reliable updates (Sleijpen & van
// der Vorst 1996) as in the kernel engine's mixed BiCGSTAB.  Shared memory
// (FP32): r, g (= p, gathered), q, y (the correction since the last
// update).  Whenever the iterated ||r|| has fallen by `delta` since the last
// true residual (or the iteration has to stop), x += y in FP64 and the true
// residual b - A x is formed with the FP64 values (S.aux); the iteration
// then goes on from it with its search direction kept.
template <bool JAC>
__device__ __forceinline__ SolveOut cg_mixed_system(ClusterEnv &E, const ClusterSystem &S,
                                                    unsigned long long budget_ns,
                                                    double delta) {
  const int RPC = E.rpc;
  float *r = reinterpret_cast<float *>(E.dyn);
  float *g = r + RPC;
  float *q = g + RPC;
  float *y = q + RPC;
  float *const *remote = reinterpret_cast<float *const *>(E.sh.remote_vec);
  const int rank = (int)E.rank, shift = E.shift, mask = E.mask;
  const int n = S.n;
  const int row0 = rank * RPC;
  const int nloc = max(0, min(RPC, n - row0));
  const int *rp = S.rp, *ci = S.ci;
  const float *val = static_cast<const float *>(S.val);
  const double *val64 = static_cast<const double *>(S.aux);
  const double *b = static_cast<const double *>(S.b);
  double *x = static_cast<double *>(S.x);
  float *dinv = static_cast<float *>(S.dinv);
  const double tol = S.tol;
  const long long maxiter = S.maxiter, miniter = S.miniter;
  const uint64_t t0 = global_timer_ns();

  cluster_jacobi_setup<float>(rp, ci, val, dinv, row0, nloc, JAC);
  // r = b - A x in FP64 (x through L2: other CTAs of the cluster write it),
  // kept in FP32; sums (z, r) and ||r64||^2; y = 0
  auto refresh = [&](double (&s2)[2]) {
    s2[0] = 0.0;
    s2[1] = 0.0;
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      double acc = 0.0;
      for (int j = __ldg(rp + row); j < __ldg(rp + row + 1); ++j)
        acc = __dadd_rn(acc, __dmul_rn(__ldg(val64 + j), __ldcg(x + __ldg(ci + j))));
      const double r64 = b[row] - acc;
      const float ri = (float)r64;
      r[i] = ri;
      const float zi = JAC ? dinv[row] * ri : ri;
      s2[0] += (double)zi * (double)ri;
      s2[1] += r64 * r64;
      y[i] = 0.0f;
    }
    env_sum<2>(E, s2);
  };
  double s2[2];
  E.cl.sync();  // dinv of every CTA
  refresh(s2);
  double rz = s2[0];
  double resid = sqrt(s2[1]);
  double rel_true = resid;
  MLSH_FOR_OWN_ROWS(i, nloc) g[i] = JAC ? dinv[row0 + i] * r[i] : r[i];
  long long it = 0;
  int status = maxiter <= 0 ? MLSH_SOLVER_MAXITER : kRunning;
  E.cl.sync();

  while (status == kRunning) {
    // q = A p, (p, q)
    double pq[1] = {0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const float qv = cluster_row_dot<float>(rp, ci, val, row0 + i, g, remote, shift, mask, rank);
      q[i] = qv;
      pq[0] += (double)g[i] * (double)qv;
    }
    env_sum<1>(E, pq);
    const float alpha = (float)(rz / pq[0]);
    // y += alpha p; r -= alpha q; (z, r), (r, r); time budget
    double s3[3] = {0.0, 0.0, 0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      y[i] = alpha * g[i] + y[i];
      const float ri = -alpha * q[i] + r[i];
      r[i] = ri;
      const float zi = JAC ? dinv[row] * ri : ri;
      s3[0] += (double)zi * (double)ri;
      s3[1] += (double)ri * (double)ri;
    }
    if (rank == 0 && threadIdx.x == 0 && global_timer_ns() - t0 > budget_ns) s3[2] = 1.0;
    env_sum<3>(E, s3);
    ++it;
    double rz_new = s3[0];
    const double rec = sqrt(s3[1]);
    const bool timeout = s3[2] > 0.0;
    if (rec < delta * rel_true || rec < tol || it >= maxiter || isnan(rec) || timeout) {
      MLSH_FOR_OWN_ROWS(i, nloc) x[row0 + i] += (double)y[i];
      E.cl.sync();  // every CTA's part of x before anyone gathers it
      refresh(s2);
      rz_new = s2[0];
      resid = sqrt(s2[1]);
      rel_true = resid;
      if (resid < tol && miniter <= it) status = MLSH_SUCCESS;
      else if (isnan(resid)) status = MLSH_SOLVER_RESIDUAL_NAN;
      else if (it >= maxiter) status = MLSH_SOLVER_MAXITER;
      else if (timeout) status = MLSH_ERR_TIMEOUT;
    }
    if (status != kRunning) break;
    const float beta = (float)(rz_new / rz);
    rz = rz_new;
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const float zi = JAC ? dinv[row0 + i] * r[i] : r[i];
      g[i] = zi + beta * g[i];
    }
    E.cl.sync();
  }
  // every x write precedes the last cluster barrier (inside env_sum)
  return SolveOut{status, it, resid};
}

// ------------------------------------------------------------- kernels --
__device__ __forceinline__ void env_init(ClusterEnv &E, void *gathered) {
  if (threadIdx.x < E.csize) {
    E.sh.remote_vec[threadIdx.x] = E.cl.map_shared_rank(gathered, threadIdx.x);
    E.sh.remote_slots[threadIdx.x] = E.cl.map_shared_rank(E.sh.slots, threadIdx.x);
  }
  E.cl.sync();
}

// Next system index from the launch's queue (rank 0 claims, all CTAs see it).
__device__ __forceinline__ unsigned long long queue_next(ClusterEnv &E, unsigned *queue) {
  if (E.rank == 0 && threadIdx.x == 0) {
    const unsigned long long idx = atomicAdd(queue, 1u);
    for (unsigned r = 0; r < E.csize; ++r) *E.cl.map_shared_rank(&E.sh.sys_idx, r) = idx;
  }
  E.cl.sync();
  return E.sh.sys_idx;
}

// KIND 0: CG, 1: BiCGSTAB, 2: mixed CG (T = float).
template <typename T, int KIND, bool JAC>
__global__ void __launch_bounds__(kClusterThreads, 1) cluster_queue_kernel(const ClusterArgs a) {
  cgs::cluster_group cl = cgs::this_cluster();
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ ClusterShared sh;
  ClusterEnv E{cl, sh, dyn, cl.num_blocks(), cl.block_rank(), a.rpc_shift, 1 << a.rpc_shift,
               (1 << a.rpc_shift) - 1, 0};
  T *gathered = reinterpret_cast<T *>(dyn) + (KIND == 1 ? 5 : 1) * E.rpc;
  env_init(E, gathered);
  while (true) {
    const unsigned long long idx = queue_next(E, a.queue);
    if (idx >= (unsigned long long)a.n_systems) break;
    ClusterSystem &S = a.systems[idx];
    SolveOut o;
    if constexpr (KIND == 0) o = cg_system<T>(E, S, JAC, a.budget_ns);
    else if constexpr (KIND == 1) o = bicgstab_system<T>(E, S, JAC, a.budget_ns);
    else o = cg_mixed_system<JAC>(E, S, a.budget_ns, a.delta);
    if (E.rank == 0 && threadIdx.x == 0) {
      S.status = o.status;
      S.iters = o.iters;
      S.resid = o.resid;
    }
  }
}

// Serving: claim the next published ring record, copy it into every CTA's
// shared memory.  Returns false when the cluster should exit (shutdown, or
// no work for idle_ns).  The wait polls with a bounded sleep.
__device__ __forceinline__ bool ring_next(ClusterEnv &E, const ServeRing &ring) {
  if (E.rank == 0 && threadIdx.x == 0) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_system> tail(*ring.tail);
    cuda::atomic_ref<int, cuda::thread_scope_system> stop(*ring.shutdown);
    unsigned long long claimed = ~0ull;
    const uint64_t t0 = global_timer_ns();
    while (true) {
      const unsigned long long h = atomicAdd(ring.head, 0ull);
      const unsigned long long t = tail.load(cuda::memory_order_acquire);
      if (h < t) {
        if (atomicCAS(ring.head, h, h + 1) == h) {
          claimed = h;
          break;
        }
        continue;
      }
      if (stop.load(cuda::memory_order_relaxed) != 0) break;
      if (global_timer_ns() - t0 > ring.idle_ns) break;
      __nanosleep(2000);
    }
    ClusterSystem rec;
    if (claimed != ~0ull) {
      // uncached word copy of the host-written record
      const volatile unsigned long long *src = reinterpret_cast<const volatile unsigned long long *>(
          ring.rec + (claimed & (ring.capacity - 1)));
      unsigned long long *dst = reinterpret_cast<unsigned long long *>(&rec);
      for (int w = 0; w < (int)(sizeof(ClusterSystem) / 8); ++w) dst[w] = src[w];
    }
    for (unsigned r = 0; r < E.csize; ++r) {
      *E.cl.map_shared_rank(&E.sh.sys_idx, r) = claimed;
      if (claimed != ~0ull) *E.cl.map_shared_rank(&E.sh.sys, r) = rec;
    }
  }
  E.cl.sync();
  return E.sh.sys_idx != ~0ull;
}

// The serving kernel: FP64, CG or BiCGSTAB per record, Jacobi or none per
// record; dynamic shared memory for BiCGSTAB's six vectors.
__global__ void __launch_bounds__(kClusterThreads, 1) cluster_serve_kernel(const ClusterArgs a) {
  cgs::cluster_group cl = cgs::this_cluster();
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ ClusterShared sh;
  ClusterEnv E{cl, sh, dyn, cl.num_blocks(), cl.block_rank(), a.rpc_shift, 1 << a.rpc_shift,
               (1 << a.rpc_shift) - 1, 0};
  // CG gathers the second vector, BiCGSTAB the sixth: both are mapped
  void *g_cg = reinterpret_cast<double *>(dyn) + E.rpc;
  void *g_bi = reinterpret_cast<double *>(dyn) + 5 * E.rpc;
  __shared__ void *remote_cg[kMaxClusterSize], *remote_bi[kMaxClusterSize];
  if (threadIdx.x < E.csize) {
    remote_cg[threadIdx.x] = cl.map_shared_rank(g_cg, threadIdx.x);
    remote_bi[threadIdx.x] = cl.map_shared_rank(g_bi, threadIdx.x);
    sh.remote_slots[threadIdx.x] = cl.map_shared_rank(sh.slots, threadIdx.x);
  }
  cl.sync();
  while (ring_next(E, a.ring)) {
    const ClusterSystem &S = sh.sys;
    const bool bicg = (S.flags & kSysBiCGSTAB) != 0;
    const bool jac = (S.flags & kSysJacobi) != 0;
    if (threadIdx.x < E.csize)
      sh.remote_vec[threadIdx.x] = bicg ? remote_bi[threadIdx.x] : remote_cg[threadIdx.x];
    __syncthreads();
    const SolveOut o = bicg ? bicgstab_system<double>(E, S, jac, a.budget_ns)
                            : cg_system<double>(E, S, jac, a.budget_ns);
    if (E.rank == 0 && threadIdx.x == 0) {
      ClusterSystem *dst = a.ring.rec + (sh.sys_idx & (a.ring.capacity - 1));
      volatile ClusterSystem *vd = dst;
      vd->status = o.status;
      vd->iters = o.iters;
      vd->resid = o.resid;
      cuda::atomic_ref<int, cuda::thread_scope_system> done(dst->done);
      done.store(1, cuda::memory_order_release);
    }
    // every CTA is done with this record before rank 0 overwrites sys
    cl.sync();
  }
}

// --------------------------------------------------------------- launcher --
namespace {

using KernelFn = void (*)(const ClusterArgs);

KernelFn cluster_kernel(int kind, int dtype, bool jac) {
  if (kind == 2) return jac ? cluster_queue_kernel<float, 2, true> : cluster_queue_kernel<float, 2, false>;
  if (kind == 0) {
    if (dtype == MLSH_F64)
      return jac ? cluster_queue_kernel<double, 0, true> : cluster_queue_kernel<double, 0, false>;
    return jac ? cluster_queue_kernel<float, 0, true> : cluster_queue_kernel<float, 0, false>;
  }
  if (dtype == MLSH_F64)
    return jac ? cluster_queue_kernel<double, 1, true> : cluster_queue_kernel<double, 1, false>;
  return jac ? cluster_queue_kernel<float, 1, true> : cluster_queue_kernel<float, 1, false>;
}

int cluster_nvec(int kind) { return kind == 0 ? 3 : (kind == 1 ? 6 : 4); }

int set_cluster_attributes() {
  static std::once_flag once;
  static int status = MLSH_SUCCESS;
  std::call_once(once, [] {
    auto set = [](KernelFn k) {
      if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kClusterMaxDynSmem) != cudaSuccess ||
          cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
              cudaSuccess) {
        cudaGetLastError();
        status = MLSH_ERR_CUDA;
      }
    };
    for (int kind = 0; kind < 2; ++kind)
      for (int dt = 0; dt < 2; ++dt)
        for (int j = 0; j < 2; ++j) set(cluster_kernel(kind, dt, j != 0));
    for (int j = 0; j < 2; ++j) set(cluster_kernel(2, MLSH_F32, j != 0));
    set(cluster_serve_kernel);
  });
  return status;
}

cudaLaunchConfig_t cluster_config(int csize, int n_clusters, size_t smem, cudaStream_t stream,
                                  cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(csize * n_clusters), 1, 1);
  cfg.blockDim = dim3(kClusterThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

}  // namespace

int cluster_rows_for(int kind, int dtype, int64_t n, int requested) {
  const int esz = dtype_size(dtype);
  int rpc = 1024;
  if (requested > 0) {
    while (rpc < requested) rpc <<= 1;
  } else {
    while ((int64_t)rpc * kMaxClusterSize < n) rpc <<= 1;
  }
  if ((int64_t)cluster_nvec(kind) * rpc * esz > kClusterMaxDynSmem) return 0;
  if ((n + rpc - 1) / rpc > kMaxClusterSize) return 0;
  return rpc;
}

int cluster_launch(const Handle &h, int kind, int dtype, bool jac, ClusterSystem *d_systems,
                   int n_systems, unsigned *d_queue, int rpc, int csize, int n_clusters,
                   double budget_s, cudaStream_t stream, double delta) {
  (void)h;
  if (set_cluster_attributes() != MLSH_SUCCESS) return MLSH_NOT_IMPL;
  int shift = 0;
  while ((1 << shift) < rpc) ++shift;
  ClusterArgs a = {};
  a.systems = d_systems;
  a.n_systems = n_systems;
  a.rpc_shift = shift;
  a.queue = d_queue;
  a.budget_ns = (unsigned long long)(budget_s * 1e9);
  a.precond = jac ? MLSH_PRECOND_JACOBI : MLSH_PRECOND_NONE;
  a.delta = delta;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(
      csize, n_clusters, (size_t)cluster_nvec(kind) * rpc * dtype_size(dtype), stream, attr);
  KernelFn k = cluster_kernel(kind, dtype, jac);
  int max_clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&max_clusters, (void *)k, &cfg) != cudaSuccess ||
      max_clusters < 1) {
    cudaGetLastError();
    return MLSH_NOT_IMPL;
  }
  if (n_clusters > max_clusters) {
    n_clusters = max_clusters;
    cfg.gridDim = dim3((unsigned)(csize * n_clusters), 1, 1);
  }
  MLSH_CUDA_TRY(cudaLaunchKernelEx(&cfg, k, a));
  return MLSH_SUCCESS;
}

int cluster_max_active(int kind, int dtype, bool jac, int rpc, int csize) {
  if (set_cluster_attributes() != MLSH_SUCCESS) return 0;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg =
      cluster_config(csize, 1, (size_t)cluster_nvec(kind) * rpc * dtype_size(dtype), nullptr,
                     attr);
  int m = 0;
  if (cudaOccupancyMaxActiveClusters(&m, (void *)cluster_kernel(kind, dtype, jac), &cfg) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return m;
}

// Serving kernel: FP64, rows per CTA kServeRows (BiCGSTAB's six vectors).
int cluster_serve_launch(const ServeRing &ring, int csize, int n_clusters, double budget_s,
                         cudaStream_t stream) {
  if (set_cluster_attributes() != MLSH_SUCCESS) return MLSH_NOT_IMPL;
  int shift = 0;
  while ((1 << shift) < kServeRows) ++shift;
  ClusterArgs a = {};
  a.rpc_shift = shift;
  a.budget_ns = (unsigned long long)(budget_s * 1e9);
  a.ring = ring;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg =
      cluster_config(csize, n_clusters, (size_t)6 * kServeRows * sizeof(double), stream, attr);
  int max_clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&max_clusters, (void *)cluster_serve_kernel, &cfg) !=
          cudaSuccess ||
      max_clusters < 1) {
    cudaGetLastError();
    return MLSH_NOT_IMPL;
  }
  if (n_clusters > max_clusters) {
    n_clusters = max_clusters;
    cfg.gridDim = dim3((unsigned)(csize * n_clusters), 1, 1);
  }
  MLSH_CUDA_TRY(cudaLaunchKernelEx(&cfg, cluster_serve_kernel, a));
  return MLSH_SUCCESS;
}

}  // namespace mlsh
