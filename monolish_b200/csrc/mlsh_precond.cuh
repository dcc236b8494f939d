// SOR / IC(0) / ILU(0) preconditioners on the device: the factorizations
// and the sparse triangular sweeps that apply them.
//
// Reference behaviour (src/equation/sor.cpp, ic.cpp, ilu.cpp and
// src/equation/kernel/{sor,ic,ilu}_kernel.hpp):
//   SOR  create: M = 1 / (omega * diag(A))                  (sor.cpp:29-32)
//        apply:  forward  y_i = (r_i - sum_{j<i} a_ij y_j) * M_i
//                backward z_i = y_i - (sum_{j>i} a_ij z_j) * M_i
//                                                (sor_kernel.hpp:42-72)
//   IC   create: IC(0) of A's lower triangle, A ~ L L^T, in A's pattern
//        apply:  L y = r, L^T z = y                 (ic_kernel.hpp, csric02
//                + two csrsv2 solves, non-unit L)
//   ILU  create: ILU(0), A ~ L U in A's pattern, L unit lower
//        apply:  L y = r, U z = y                   (ilu_kernel.hpp, csrilu02
//                + two csrsv2 solves)
// The reference runs IC and ILU through cuSPARSE; here both the
// factorizations and the sweeps are this library's own kernels.
//
// The sweeps are synchronization-free (Liu et al., "A synchronization-free
// algorithm for parallel sparse triangular solves", Euro-Par 2016, here in
// row-oriented CSR form) over a level schedule: rows are grouped in blocks
// of 32 consecutive rows; at setup each block's dependency blocks (those its
// rows reference outside the block) and its level in the block DAG are
// computed, and the blocks are ordered by level.  One warp per block; an
// atomic ticket hands the blocks out in that order, so every block a warp
// waits on belongs to a warp that is already running, and the warps
// resident at any time hold a band of consecutive levels -- the wavefront
// -- rather than a band of consecutive rows.  A warp's lanes wait on the
// block's dependency flags in parallel (GPU-scope acquire), load the values
// their rows need from outside the block, resolve the dependencies inside
// the block as a 32-step chain of register shuffles, publish the 32 results
// and set the block's flag.  Flags carry a launch epoch derived from the
// ticket counter, so they never need clearing and graph replays stay valid.
// Every wait is bounded; a warp that gives up records MLSH_ERR_TIMEOUT and
// still publishes its flag, so no other warp waits on it for long.  The
// factorizations use the same schedule with one warp per row.  A system
// whose solution vector and schedule fit in 200 KB of shared memory is
// swept by one CTA instead: its warps take each level's blocks with a CTA
// barrier between levels, so a dependency costs a barrier rather than a
// round trip through L2 between SMs.
#pragma once
#include "mlsh_internal.cuh"

namespace mlsh {

enum SweepMode {
  kSorFwd = 0,   // y_i = (r_i - sum_lower a y) * scale_i
  kUnitFwd = 1,  // y_i =  r_i - sum_lower a y
  kDiagFwd = 2,  // y_i = (r_i - sum_lower a y) / a_ii
  kSorBwd = 3,   // z_i =  y_i - (sum_upper a z) * scale_i
  kDiagBwd = 4,  // z_i = (y_i - sum_upper a z) / a_ii
};

// One triangular sweep over a CRS pattern with sorted rows: lo_end[i] is
// the first entry of row i with column >= i, up_beg[i] the first with
// column > i (up_beg[i] > lo_end[i] iff the diagonal is stored).
struct Sweep {
  const int *rp = nullptr;
  const int *ci = nullptr;
  const void *val = nullptr;
  const int *lo_end = nullptr;
  const int *up_beg = nullptr;
  const void *scale = nullptr;  // SOR modes: per-row multiplier
  int mode = kSorFwd;
  // schedule: blocks in level order, each block's dependency blocks (CSR)
  const int *order = nullptr;
  const int *dep_off = nullptr;
  const int *dep_ids = nullptr;
};

// A level schedule of the row blocks for one sweep direction.
struct Schedule {
  int *order = nullptr;    // nb block ids, by level
  int *dep_off = nullptr;  // nb + 1
  int *dep_ids = nullptr;  // dependency blocks of each block
  int *level_off = nullptr;  // levels + 1: where each level starts in order
  int levels = 0;          // length of the longest dependency chain
  long long deps = 0;      // total dependency entries
  int width = 0;           // most blocks in one level
  // single-CTA ring sweep: each block's matrix-only row state, in level
  // order (one record per block), and the shared-memory ring's slot count
  // (0: the sweep does not take the ring form)
  void *rec = nullptr;
  int ring = 0;
};

constexpr unsigned kDefaultWaitPolls = 1u << 22;  // a few seconds of polling

struct Precond {
  Handle *handle = nullptr;
  const CsrPlan *plan = nullptr;
  int kind = 0;   // MLSH_PRECOND_SOR / _IC / _ILU
  int dtype = MLSH_F64;
  int n = 0, nnz = 0;
  unsigned nb = 0;  // row blocks of 32
  Sweep fwd, bwd;
  // owned device buffers
  int *lo_end = nullptr, *up_beg = nullptr;  // A's pattern
  void *fval = nullptr;                      // IC / ILU factor, A's pattern
  int *rp_t = nullptr, *ci_t = nullptr;      // IC: transpose of the factor
  void *val_t = nullptr;
  int *lo_t = nullptr, *up_t = nullptr;
  void *scale = nullptr;  // SOR: per-row multiplier
  void *tmp = nullptr;    // the intermediate vector of apply
  Schedule sfwd, sbwd;    // lower / upper sweep schedules
  unsigned long long *ticket = nullptr;
  unsigned *flags = nullptr;  // nb block flags
  long long pivot = -1;       // first zero pivot, -1 if none
  int structural = 0;         // 1: that row has no stored diagonal
  unsigned wait_polls = kDefaultWaitPolls;  // polls per sweep wait (opts->wait_polls)
};

// out = sweep(rhs) (backward = the upper sweep, blocks from the last row
// up).  `done` (optional) skips the launch once a solve has finished.
cudaError_t sweep_launch(const Precond &pc, const Sweep &sw, bool backward, const void *rhs,
                         void *out, const int *done, int *err, cudaStream_t s);
// z = M^{-1} r: the forward sweep into pc.tmp, the backward sweep into z.
cudaError_t precond_apply_launch(const Precond &pc, const void *r, void *z, const int *done,
                                 int *err, cudaStream_t s);

// Builds a preconditioner of `kind` for the plan's matrix on h's stream.
// solver_scale: SOR only, the scaling of the SOR solver's own sweep
// (omega / diag(A), sor.cpp:112-115) instead of the preconditioner's.
int precond_build(Handle &h, const CsrPlan &p, int kind, double omega, bool solver_scale,
                  Precond &out);
void precond_release(Precond &pc);

// Drops solver graphs that captured this preconditioner (mlsh_krylov.cu).
void purge_precond_graphs(Handle &h, const Precond *pc);

}  // namespace mlsh

struct mlsh_precond_s {
  mlsh::Precond p;
};
