// Cluster-resident CG / BiCGSTAB kernels and their launcher (see
// mlsh_cluster.cuh for the design).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "mlsh_cluster.cuh"
#include "mlsh_core.cuh"

namespace mlsh {

namespace cgs = cooperative_groups;

// Shared state of one CTA of the cluster engine.
struct ClusterShared {
  double slots[2 * 3 * kMaxClusterSize];  // [parity][k][rank]
  double red_warp[32 * 3];
  void *remote_vec[kMaxClusterSize];      // gathered-vector slice of each CTA
  double *remote_slots[kMaxClusterSize];
  unsigned sys_idx;
};

// Thread's k-th own row (local index) of the CTA's slice.
#define MLSH_FOR_OWN_ROWS(i, nloc) \
  for (int i = (int)threadIdx.x; i < (nloc); i += kClusterThreads)

template <typename T, bool JAC>
__device__ __forceinline__ void cluster_jacobi_setup(const int *rp, const int *ci, const T *val,
                                                     T *dinv, int row0, int nloc) {
  if constexpr (JAC) {
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      T d = T(0);
      for (int j = __ldg(rp + row); j < __ldg(rp + row + 1); ++j)
        if (__ldg(ci + j) == row) d = __ldg(val + j);
      dinv[row] = T(1) / d;
    }
  }
}

__device__ __forceinline__ unsigned cluster_next_system(ClusterShared &sh, unsigned *queue,
                                                        cgs::cluster_group &cl) {
  if (cl.block_rank() == 0 && threadIdx.x == 0) {
    const unsigned idx = atomicAdd(queue, 1u);
    for (unsigned r = 0; r < cl.num_blocks(); ++r) *cl.map_shared_rank(&sh.sys_idx, r) = idx;
  }
  cl.sync();
  return sh.sys_idx;
}

// ------------------------------------------------------------------- CG --
template <typename T, bool JAC>
__global__ void __launch_bounds__(kClusterThreads, 1) cluster_cg_kernel(const ClusterArgs a) {
  cgs::cluster_group cl = cgs::this_cluster();
  const unsigned csize = cl.num_blocks();
  const unsigned rank = cl.block_rank();
  const int shift = a.rpc_shift, RPC = 1 << shift, mask = RPC - 1;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ ClusterShared sh;
  T *r = reinterpret_cast<T *>(dyn);
  T *g = r + RPC;  // p, gathered by the SpMV
  T *q = g + RPC;
  if (threadIdx.x < csize) {
    sh.remote_vec[threadIdx.x] = cl.map_shared_rank(g, threadIdx.x);
    sh.remote_slots[threadIdx.x] = cl.map_shared_rank(sh.slots, threadIdx.x);
  }
  cl.sync();
  T *const *remote = reinterpret_cast<T *const *>(sh.remote_vec);
  int parity = 0;

  while (true) {
    const unsigned idx = cluster_next_system(sh, a.queue, cl);
    if (idx >= (unsigned)a.n_systems) break;
    ClusterSystem &S = a.systems[idx];
    const int n = S.n;
    const int row0 = (int)rank * RPC;
    const int nloc = max(0, min(RPC, n - row0));
    const int *rp = S.rp, *ci = S.ci;
    const T *val = static_cast<const T *>(S.val);
    const T *b = static_cast<const T *>(S.b);
    T *x = static_cast<T *>(S.x);
    T *dinv = static_cast<T *>(S.dinv);
    const double tol = S.tol;
    const long long maxiter = S.maxiter, miniter = S.miniter;
    const uint64_t t0 = global_timer_ns();

    cluster_jacobi_setup<T, JAC>(rp, ci, val, dinv, row0, nloc);
    MLSH_FOR_OWN_ROWS(i, nloc) g[i] = x[row0 + i];
    cl.sync();
    // r = b - A x0 (cg.cpp:39-40), z = M r, p = z (cg.cpp:43-44)
    double acc[3] = {0.0, 0.0, 0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      const T qv = cluster_row_dot<T>(rp, ci, val, row, g, remote, shift, mask, (int)rank);
      const T ri = b[row] - qv;
      r[i] = ri;
      const T zi = JAC ? dinv[row] * ri : ri;
      q[i] = zi;
      acc[0] += (double)zi * (double)ri;
      acc[1] += (double)ri * (double)ri;
    }
    {
      double s2[2] = {acc[0], acc[1]};
      cluster_sum<2>(s2, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
      parity ^= 1;
      acc[0] = s2[0];
      acc[1] = s2[1];
    }
    double rz = acc[0], rr = acc[1];
    MLSH_FOR_OWN_ROWS(i, nloc) g[i] = q[i];
    long long it = 0;
    int status = maxiter <= 0 ? MLSH_SOLVER_MAXITER : kRunning;
    double resid = cl_resid<T>(rr);
    cl.sync();

    while (status == kRunning) {
      // q = A p, (p, q)
      double pq[1] = {0.0};
      MLSH_FOR_OWN_ROWS(i, nloc) {
        const T qv = cluster_row_dot<T>(rp, ci, val, row0 + i, g, remote, shift, mask, (int)rank);
        q[i] = qv;
        pq[0] += (double)g[i] * (double)qv;
      }
      cluster_sum<1>(pq, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
      parity ^= 1;
      const T alpha = (T)(rz / pq[0]);
      // x += alpha p; r -= alpha q; (z, r), (r, r); time budget
      double s3[3] = {0.0, 0.0, 0.0};
      MLSH_FOR_OWN_ROWS(i, nloc) {
        const int row = row0 + i;
        const T pi = g[i], qi = q[i];
        x[row] = alpha * pi + x[row];
        const T ri = -alpha * qi + r[i];
        r[i] = ri;
        const T zi = JAC ? dinv[row] * ri : ri;
        s3[0] += (double)zi * (double)ri;
        s3[1] += (double)ri * (double)ri;
      }
      if (rank == 0 && threadIdx.x == 0 && global_timer_ns() - t0 > a.budget_ns) s3[2] = 1.0;
      cluster_sum<3>(s3, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
      parity ^= 1;
      rr = s3[1];
      ++it;
      resid = cl_resid<T>(rr);
      if (rank == 0 && threadIdx.x == 0 && S.hist != nullptr && it <= S.hist_cap)
        S.hist[it - 1] = resid;
      if (resid < tol && miniter <= it) status = MLSH_SUCCESS;
      else if (isnan(resid)) status = MLSH_SOLVER_RESIDUAL_NAN;
      else if (it >= maxiter) status = MLSH_SOLVER_MAXITER;
      else if (s3[2] > 0.0) status = MLSH_ERR_TIMEOUT;
      if (status != kRunning) break;
      const T beta = (T)(s3[0] / rz);
      rz = s3[0];
      // p = z + beta p (cg.cpp:59)
      MLSH_FOR_OWN_ROWS(i, nloc) {
        const T zi = JAC ? dinv[row0 + i] * r[i] : r[i];
        g[i] = zi + beta * g[i];
      }
      cl.sync();
    }
    if (rank == 0 && threadIdx.x == 0) {
      S.status = status;
      S.iters = it;
      S.resid = resid;
    }
  }
}

// ------------------------------------------------------------- BiCGSTAB --
template <typename T, bool JAC>
__global__ void __launch_bounds__(kClusterThreads, 1)
    cluster_bicgstab_kernel(const ClusterArgs a) {
  cgs::cluster_group cl = cgs::this_cluster();
  const unsigned csize = cl.num_blocks();
  const unsigned rank = cl.block_rank();
  const int shift = a.rpc_shift, RPC = 1 << shift, mask = RPC - 1;
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ ClusterShared sh;
  T *r = reinterpret_cast<T *>(dyn);
  T *p = r + RPC;
  T *v = p + RPC;
  T *s = v + RPC;
  T *t = s + RPC;
  T *g = t + RPC;  // p-hat, then s-hat: gathered by the SpMVs
  if (threadIdx.x < csize) {
    sh.remote_vec[threadIdx.x] = cl.map_shared_rank(g, threadIdx.x);
    sh.remote_slots[threadIdx.x] = cl.map_shared_rank(sh.slots, threadIdx.x);
  }
  cl.sync();
  T *const *remote = reinterpret_cast<T *const *>(sh.remote_vec);
  int parity = 0;

  while (true) {
    const unsigned idx = cluster_next_system(sh, a.queue, cl);
    if (idx >= (unsigned)a.n_systems) break;
    ClusterSystem &S = a.systems[idx];
    const int n = S.n;
    const int row0 = (int)rank * RPC;
    const int nloc = max(0, min(RPC, n - row0));
    const int *rp = S.rp, *ci = S.ci;
    const T *val = static_cast<const T *>(S.val);
    const T *b = static_cast<const T *>(S.b);
    T *x = static_cast<T *>(S.x);
    T *dinv = static_cast<T *>(S.dinv);
    T *r0 = static_cast<T *>(S.aux);
    const double tol = S.tol;
    const long long maxiter = S.maxiter, miniter = S.miniter;
    const uint64_t t0 = global_timer_ns();

    cluster_jacobi_setup<T, JAC>(rp, ci, val, dinv, row0, nloc);
    MLSH_FOR_OWN_ROWS(i, nloc) g[i] = x[row0 + i];
    cl.sync();
    // r = b - A x, r0 = r (bicgstab.cpp:47-51)
    double s2[2] = {0.0, 0.0};
    MLSH_FOR_OWN_ROWS(i, nloc) {
      const int row = row0 + i;
      const T ri = b[row] - cluster_row_dot<T>(rp, ci, val, row, g, remote, shift, mask, (int)rank);
      r[i] = ri;
      r0[row] = ri;
      s2[0] += (double)ri * (double)ri;
      s2[1] += (double)ri * (double)ri;
    }
    cluster_sum<2>(s2, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
    parity ^= 1;
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
        g[i] = JAC ? dinv[row0 + i] * pi : pi;
      }
      cl.sync();
      // v = A p-hat; alpha = rho / (v, r0)
      double vr[1] = {0.0};
      MLSH_FOR_OWN_ROWS(i, nloc) {
        const int row = row0 + i;
        const T vv = cluster_row_dot<T>(rp, ci, val, row, g, remote, shift, mask, (int)rank);
        v[i] = vv;
        vr[0] += (double)vv * (double)r0[row];
      }
      cluster_sum<1>(vr, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
      parity ^= 1;
      const T alpha = (T)(rho / vr[0]);
      alpha_d = (double)alpha;
      // s = r - alpha v; s-hat = M s
      MLSH_FOR_OWN_ROWS(i, nloc) {
        const T si = -alpha * v[i] + r[i];
        s[i] = si;
        g[i] = JAC ? dinv[row0 + i] * si : si;
      }
      cl.sync();
      // t = A s-hat; omega = (t, s) / (t, t)
      double tw[2] = {0.0, 0.0};
      MLSH_FOR_OWN_ROWS(i, nloc) {
        const T tv = cluster_row_dot<T>(rp, ci, val, row0 + i, g, remote, shift, mask, (int)rank);
        t[i] = tv;
        tw[0] += (double)tv * (double)s[i];
        tw[1] += (double)tv * (double)tv;
      }
      cluster_sum<2>(tw, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
      parity ^= 1;
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
        const T di = JAC ? dinv[row] : T(1);
        const T ph = JAC ? di * p[i] : p[i];
        const T shh = JAC ? di * s[i] : s[i];
        T xi = alpha * ph + x[row];
        xi = omega * shh + xi;
        x[row] = xi;
        const T ri = -omega * t[i] + s[i];
        r[i] = ri;
        s3[0] += (double)ri * (double)r0[row];
        s3[1] += (double)ri * (double)ri;
      }
      if (rank == 0 && threadIdx.x == 0 && global_timer_ns() - t0 > a.budget_ns) s3[2] = 1.0;
      cluster_sum<3>(s3, sh.red_warp, sh.remote_slots, sh.slots, parity, csize, rank, cl);
      parity ^= 1;
      rr = s3[1];
      ++it;
      resid = cl_resid<T>(rr);
      if (rank == 0 && threadIdx.x == 0 && S.hist != nullptr && it <= S.hist_cap)
        S.hist[it - 1] = resid;
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
    if (rank == 0 && threadIdx.x == 0) {
      S.status = status;
      S.iters = it;
      S.resid = resid;
    }
  }
}

// --------------------------------------------------------------- launcher --
namespace {

using KernelFn = void (*)(const ClusterArgs);

KernelFn cluster_kernel(int kind, int dtype, bool jac) {
  if (kind == 0) {
    if (dtype == MLSH_F64) return jac ? cluster_cg_kernel<double, true> : cluster_cg_kernel<double, false>;
    return jac ? cluster_cg_kernel<float, true> : cluster_cg_kernel<float, false>;
  }
  if (dtype == MLSH_F64)
    return jac ? cluster_bicgstab_kernel<double, true> : cluster_bicgstab_kernel<double, false>;
  return jac ? cluster_bicgstab_kernel<float, true> : cluster_bicgstab_kernel<float, false>;
}

int cluster_nvec(int kind) { return kind == 0 ? 3 : 6; }

int set_cluster_attributes() {
  static std::once_flag once;
  static int status = MLSH_SUCCESS;
  std::call_once(once, [] {
    for (int kind = 0; kind < 2; ++kind)
      for (int dt = 0; dt < 2; ++dt)
        for (int j = 0; j < 2; ++j) {
          KernelFn k = cluster_kernel(kind, dt, j != 0);
          if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kClusterMaxDynSmem) != cudaSuccess ||
              cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                  cudaSuccess) {
            cudaGetLastError();
            status = MLSH_ERR_CUDA;
          }
        }
  });
  return status;
}

}  // namespace

int cluster_rows_for(int kind, int dtype, int64_t n, int requested) {
  const int esz = dtype_size(dtype);
  int rpc = 1024;
  if (requested > 0) {
    rpc = 1024;
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
                   double budget_s, cudaStream_t stream) {
  if (set_cluster_attributes() != MLSH_SUCCESS) return MLSH_NOT_IMPL;
  int shift = 0;
  while ((1 << shift) < rpc) ++shift;
  ClusterArgs a;
  a.systems = d_systems;
  a.n_systems = n_systems;
  a.rpc_shift = shift;
  a.queue = d_queue;
  a.budget_ns = (unsigned long long)(budget_s * 1e9);
  a.precond = jac ? MLSH_PRECOND_JACOBI : MLSH_PRECOND_NONE;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(csize * n_clusters), 1, 1);
  cfg.blockDim = dim3(kClusterThreads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)cluster_nvec(kind) * rpc * dtype_size(dtype);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
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
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)csize, 1, 1);
  cfg.blockDim = dim3(kClusterThreads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)cluster_nvec(kind) * rpc * dtype_size(dtype);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int m = 0;
  if (cudaOccupancyMaxActiveClusters(&m, (void *)cluster_kernel(kind, dtype, jac), &cfg) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return m;
}

}  // namespace mlsh
