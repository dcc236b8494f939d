// Cluster-resident Krylov solves for small and medium systems.
//
// One thread-block cluster (up to 16 CTAs on B200, 1024 threads each) runs
// a whole CG or BiCGSTAB solve in one launch: no kernel boundary, no host
// round trip and no grid-wide barrier per iteration.
//   * CTA `rank` owns rows [rank*RPC, (rank+1)*RPC) (RPC a power of two);
//     its slices of the iteration vectors live in its shared memory.
//   * The SpMV reads the gathered vector (p, or p-hat / s-hat) of the other
//     CTAs directly from their shared memory (distributed shared memory).
//   * A global sum is one CTA-wide reduction, a broadcast of the CTA's
//     partial into every CTA's shared memory, and one barrier.cluster;
//     afterwards every CTA adds the same partials in rank order, so all
//     CTAs hold bit-identical scalars and take identical branches.
//   * Recurrences, stopping rule and breakdown checks are those of
//     src/equation/cg.cpp:13-86 and src/equation/bicgstab.cpp:13-135;
//     SpMV rows are summed in row order with separately rounded products
//     (the reference's row loop, crs_matvec.hpp:101-108).
//   * A wall-clock budget is folded into the per-iteration reduction so a
//     solve that does not terminate ends with MLSH_ERR_TIMEOUT.
// The same per-system code serves the batched solver (clusters take
// systems from a queue until it is empty) and the solve server (clusters
// claim records from a ring that the host fills while the kernel runs).
#pragma once
#include <cooperative_groups.h>

#include "mlsh_internal.cuh"
#include "mlsh_ptx.cuh"
#include "mlsh_reduce.cuh"

namespace mlsh {

constexpr int kClusterThreads = 1024;
constexpr int kMaxClusterSize = 16;
// Dynamic shared memory of one CTA: 3 vectors x 8192 doubles (CG) or
// 6 vectors x 4096 doubles (BiCGSTAB); twice the rows in FP32.
constexpr int kClusterMaxDynSmem = 196608;
// Wall-clock budget of one cluster solve.
constexpr double kClusterBudgetSeconds = 60.0;
// A solve's budget: opts->time_limit when set, else the default.
inline double cluster_budget(const mlsh_solver_opts *opts) {
  return opts && opts->time_limit > 0.0 ? opts->time_limit : kClusterBudgetSeconds;
}
// AUTO engine: longest maxiter sent to the single-launch cluster engine.
constexpr long long kClusterMaxIterAuto = 2000000;
// Serving kernel: FP64 rows per CTA (BiCGSTAB's six vectors fit).
constexpr int kServeRows = 4096;

// One linear system for the cluster engine.
struct ClusterSystem {
  const int *rp;     // row_ptr [n+1] (0-based within the system)
  const int *ci;     // column indices (0-based within the system)
  const void *val;   // values (dtype of the launch)
  const void *b;     // right-hand side [n]
  void *x;           // initial guess in, solution out [n]
  void *dinv;        // workspace [n]: inverse diagonal (Jacobi)
  void *aux;         // workspace [n]: BiCGSTAB r0
  int n;
  int flags;         // serving ring: bit 0 BiCGSTAB, bit 1 Jacobi
  double tol;        // absolute ||r|| threshold
  long long maxiter;
  long long miniter;
  double *hist;      // optional residual history [hist_cap]
  long long hist_cap;
  // results
  int status;
  int done;          // serving ring: set (system scope, release) when final
  long long iters;
  double resid;
};

constexpr int kSysBiCGSTAB = 1;
constexpr int kSysJacobi = 2;

// Serving ring: records in host-mapped memory, published by the host.
struct ServeRing {
  ClusterSystem *rec;            // [capacity], host memory mapped into the device
  unsigned long long *tail;      // host-mapped: records published so far
  unsigned long long *head;      // device: records claimed so far
  int *shutdown;                 // host-mapped: nonzero asks the kernel to exit
  unsigned capacity;             // power of two
  unsigned long long idle_ns;    // clusters exit after this long without work
};
static_assert(sizeof(ClusterSystem) % 8 == 0, "records are copied as 8-byte words");

struct ClusterArgs {
  ClusterSystem *systems;
  int n_systems;
  int rpc_shift;            // rows per CTA = 1 << rpc_shift
  unsigned *queue;          // next system index (zero before the launch)
  unsigned long long budget_ns;
  int precond;              // MLSH_PRECOND_*
  ServeRing ring;           // used by the serving kernel only
  double delta;             // mixed CG: refresh once ||r|| fell by this factor
};

template <typename T>
__device__ __forceinline__ T mul_rn(T a, T b) {
  if constexpr (sizeof(T) == 8) return __dmul_rn(a, b);
  else return __fmul_rn(a, b);
}
template <typename T>
__device__ __forceinline__ T add_rn(T a, T b) {
  if constexpr (sizeof(T) == 8) return __dadd_rn(a, b);
  else return __fadd_rn(a, b);
}

// One entry of the gathered vector: this CTA's own slice through ld.shared,
// another CTA's through distributed shared memory.
template <typename T>
__device__ __forceinline__ T cluster_gather(int c, const T *local, T *const *remote, int shift,
                                            int mask, int rank) {
  const int owner = c >> shift;
  return owner == rank ? local[c & mask] : remote[owner][c & mask];
}

// y_i = sum_j a_ij g_j over row i, g gathered from the cluster's CTAs.
template <typename T>
__device__ __forceinline__ T cluster_row_dot(const int *__restrict__ rp, const int *__restrict__ ci,
                                             const T *__restrict__ val, int row, const T *local,
                                             T *const *remote, int shift, int mask, int rank) {
  const int j0 = __ldg(rp + row), j1 = __ldg(rp + row + 1);
  T sum = T(0);
  int j = j0;
  for (; j + 3 < j1; j += 4) {
    const int c0 = __ldg(ci + j), c1 = __ldg(ci + j + 1), c2 = __ldg(ci + j + 2),
              c3 = __ldg(ci + j + 3);
    const T v0 = __ldg(val + j), v1 = __ldg(val + j + 1), v2 = __ldg(val + j + 2),
            v3 = __ldg(val + j + 3);
    const T g0 = cluster_gather(c0, local, remote, shift, mask, rank);
    const T g1 = cluster_gather(c1, local, remote, shift, mask, rank);
    const T g2 = cluster_gather(c2, local, remote, shift, mask, rank);
    const T g3 = cluster_gather(c3, local, remote, shift, mask, rank);
    sum = add_rn(sum, mul_rn(v0, g0));
    sum = add_rn(sum, mul_rn(v1, g1));
    sum = add_rn(sum, mul_rn(v2, g2));
    sum = add_rn(sum, mul_rn(v3, g3));
  }
  for (; j < j1; ++j) {
    const int c = __ldg(ci + j);
    sum = add_rn(sum, mul_rn(__ldg(val + j), cluster_gather(c, local, remote, shift, mask, rank)));
  }
  return sum;
}

// Cluster-wide sum of NR doubles.  `slots` is this CTA's
// [2][kClusterMaxNR][16] buffer; `remote_slots[r]` the same buffer in CTA r.
// `parity` alternates between calls (two buffers make one barrier per
// reduction enough: a slot is rewritten only after a later barrier that every
// reader has passed).  Each parity owns a fixed kClusterMaxNR-wide half
// whatever NR is, so consecutive reductions of different widths never share
// a slot (with a stride of NR, a one-value reduction at parity 1 and the next
// three-value one at parity 0 would: a CTA ahead could overwrite a slot that
// another CTA has yet to read).
constexpr int kClusterMaxNR = 3;
template <int NR>
__device__ __forceinline__ void cluster_sum(double (&v)[NR], double *red_warp,
                                            double *const *remote_slots, double *slots,
                                            int parity, unsigned csize, unsigned rank,
                                            cooperative_groups::cluster_group &cl) {
  static_assert(kClusterThreads == 32 * 32, "one warp partial per lane of warp 0");
  static_assert(NR >= 1 && NR <= kClusterMaxNR, "slots hold kClusterMaxNR values per parity");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) red_warp[warp * NR + k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    // warp 0: lane l holds warp l's partial; xor tree -> CTA sum in every
    // lane; lane r stores it into CTA r's slot for this rank
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double s = warp_sum(red_warp[lane * NR + k]);
      if ((unsigned)lane < csize)
        remote_slots[lane][(parity * kClusterMaxNR + k) * kMaxClusterSize + rank] = s;
    }
  }
  cl.sync();
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double *sl = slots + (parity * kClusterMaxNR + k) * kMaxClusterSize;
    double part[kMaxClusterSize];
#pragma unroll
    for (int r = 0; r < kMaxClusterSize; ++r) part[r] = (unsigned)r < csize ? sl[r] : 0.0;
    double s = 0.0;
#pragma unroll
    for (int r = 0; r < kMaxClusterSize; ++r) s += part[r];
    v[k] = s;
  }
}

template <typename T>
__device__ __forceinline__ double cl_resid(double rr) {
  if constexpr (sizeof(T) == 8) return sqrt(rr);
  else return (double)sqrtf((float)rr);
}

}  // namespace mlsh
