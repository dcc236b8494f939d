// Internal definitions shared by the CUDA translation units: the handle and
// plan objects behind the opaque C types, the device solver-state block,
// launch geometry constants and error plumbing.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/mlsh.h"

namespace mlsh {

// ----------------------------------------------------------- geometry ----
// SpMV row tiles: at most kTileRows rows and kTileNnz nonzeros each, so one
// consumer thread owns one row of a tile and a tile's values+indices fit a
// pipeline stage in shared memory.  Rows longer than kTileNnz are split into
// chunks of kTileNnz nonzeros that are summed by a second step.
constexpr int kTileRows = 256;
constexpr int kTileNnz = 1792;  // = 256 rows x 7 nonzeros (7-point stencil)
// Rows longer than this get tiles of their own (chunks of kTileNnz), summed
// by the whole CTA; shorter rows are summed by the warp that owns them.
// (A lower threshold was measured slower on Zipf-law rows: one-row tiles
// cost a CTA barrier each.)
constexpr int kLongRow = kTileNnz;
constexpr int kConsumers = 256;  // consumer threads per CTA (8 warps)
constexpr int kSpmvThreads = kConsumers + 32;  // + one producer warp
constexpr int kShortRow = 8;     // thread-per-row sums load x in batches of this many
// Rows up to a plan's short-row limit (kShortRow, 2 kShortRow or 4 kShortRow,
// picked by the autotuner) are summed by one thread in row order.
constexpr int kMaxShortRow = 4 * kShortRow;
constexpr int kDefaultSpmvVariant = 2;  // until the plan is autotuned

// Elementwise / reduction kernels.
constexpr int kVecThreads = 256;
constexpr int kMaxVecBlocksPerSm = 8;
constexpr int kMaxPartialBlocks = 4096;  // upper bound of any reduction grid
constexpr int kMaxRed = 4;               // reduction values per kernel

// Device waits give up after this long and report MLSH_ERR_TIMEOUT.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// Solver status while iterating.
constexpr int kRunning = 1;

// --------------------------------------------------------- tile record ---
// Normal tile: rows [row_begin, row_end), nonzeros [nnz_begin, nnz_end).
// Chunk of a long row: row_begin = row, row_end = -(long_index + 1),
// pad[0] = the row's chunk count.
// short_only: every row of a normal tile has at most kShortRow entries.
struct __align__(16) Tile {
  int row_begin;
  int row_end;
  int nnz_begin;
  int nnz_end;
  int short_only;
  int pad[3];
};

struct LongRow {
  int row;
  int first_slot;  // index of chunk 0 in the plan's chunk-partial array
  int n_chunks;
  int pad;
};

// ------------------------------------------------- device solver state ---
// One block per handle; written only by the last CTA of each kernel (after
// every other CTA has finished reading it) or by single-thread kernels.
struct SolverState {
  // scalars of the recurrences (double for both dtypes)
  double rz;       // CG: (z, r) of the current iterate
  double rz_new;   // CG: (z, r) after the update
  double pq;       // CG: (p, A p)
  double rr;       // (r, r)
  double rho;      // BiCGSTAB: (r, r0)
  double rho_old;
  double alpha;
  double omega;
  double vr0;      // BiCGSTAB: (v, r0)
  double ts;       // BiCGSTAB: (t, s)
  double tt;       // BiCGSTAB: (t, t)
  double resid;    // ||r||_2 as the stopping rule sees it
  double tol;      // absolute tolerance
  double pad0;
  long long iter;  // iterations completed
  long long maxiter;
  long long miniter;
  int status;      // kRunning or a final MLSH_* code
  int done;        // 1 once status is final
  int error;       // MLSH_ERR_TIMEOUT if a device wait gave up
  int pad1;
  double *hist;    // optional residual history (device), hist_cap entries
  long long hist_cap;
  // mixed precision with reliable updates: FP32 iteration vectors hold the
  // FP64 quantities divided by `scale`; x and the true residual are FP64
  double scale;
  double rr64;      // ||b - A x||^2 of the last FP64 residual
  double rel_true;  // true ||r|| at the last update
  double delta;     // update once the iterated ||r|| < delta * rel_true
  long long outer;  // FP64 residual evaluations after the first
  int upd;          // 1: the update kernels run at the start of the next pass
  int noupd;        // 1 - upd (the update kernels' skip flag)
  int first;        // 1: the next iteration starts a fresh Krylov space
  int pending;      // status the iteration ended with, applied after the update
};

// ------------------------------------------------------------- objects ---
struct Handle {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  // reduction scratch: per-block partials + one arrival counter per slot
  double *partials = nullptr;    // kMaxPartialBlocks * kMaxRed doubles
  unsigned *counters = nullptr;  // 8 counters, zero between kernels
  double *scalars = nullptr;     // 8 doubles of device results
  SolverState *state = nullptr;
  SolverState *host_state = nullptr;  // pinned mirror
  double *host_scalars = nullptr;     // pinned
  int *err_flag = nullptr;            // device: nonzero after a timeout
  cudaStream_t capture_stream = nullptr;  // private stream for graph capture
  void *ws = nullptr;                 // solver work vectors
  size_t ws_bytes = 0;
  void *graph_cache = nullptr;        // instantiated solver graphs
  double *hist = nullptr;             // residual history buffer (device)
  long long hist_cap = 0;
  void *host_cluster = nullptr;       // pinned record for the cluster engine
};

// Offset-slot layout of an FP32 copy (mlsh_slots.cu): the matrix uses at
// most kMaxSlots distinct column offsets (col - row), held once in `offs`;
// rows are cut into slices of kSlotRows, and a slice is one contiguous
// record of slot_rec_bytes(K) bytes:
//   uint8 mask[kSlotRows]     bit k = the row has an entry at offs[k]
//   float vals[K][kSlotRows]  values slot-major (0 where absent)
// so one bulk copy moves a slice into shared memory.
constexpr int kSlotRows = 256;
constexpr int kMaxSlots = 8;
constexpr int kSlotHeadBytes = kSlotRows;  // the mask; a multiple of 16
__host__ __device__ constexpr int slot_rec_bytes(int K) {
  return kSlotHeadBytes + 4 * kSlotRows * K;
}
// The SpMV moves kSlotGroup consecutive slices per pipeline stage: their
// records, and x as a few windows -- offsets closer than kSlotMergeGap share
// one window x[R0 + lo .. R0 + hi + kSlotGroup * kSlotRows), R0 the stage's
// first row.  (Two slices: small enough stages for four of them per CTA and
// two CTAs per SM.)
constexpr int kSlotGroup = 2;
constexpr int kSlotMergeGap = 1024;
constexpr int kMaxSlotWin = kMaxSlots + 1;  // the slots' windows + the diagonal's
constexpr int kMaxSlotStages = 4;
struct SlotFormat {
  unsigned char *recs = nullptr;  // n_slices records
  int offs[kMaxSlots] = {0, 0, 0, 0, 0, 0, 0, 0};  // ascending; the first K are used
  int K = 0;                      // stored slots
  int unit = 0;                   // 1: every diagonal value is exactly 1 and not stored
  int n_slices = 0;
  // stage plan
  int n_win = 0;
  int win_lo[kMaxSlotWin] = {};   // window start, relative to the stage's first row
  int win_len[kMaxSlotWin] = {};  // window length in elements
  int win_off[kMaxSlotWin] = {};  // byte offset of the window in a stage
  int slot_win[kMaxSlots] = {};   // the window holding slot k's x values
  int diag_win = -1;              // the window holding x_i (unit diagonal)
  int w_off = 0;                  // byte offset of the dot weights' runs in a stage
  int stage_bytes = 0;
  int stages = 0;
  int grid_per_sm = 0;            // CTAs per SM of the launch
  int64_t bytes() const { return (int64_t)n_slices * slot_rec_bytes(K); }
};

struct CsrPlan {
  Handle *handle = nullptr;
  int n_rows = 0, n_cols = 0, nnz = 0;
  int dtype = MLSH_F64;
  const int *row_ptr = nullptr;
  const int *col_ind = nullptr;
  const void *val = nullptr;
  // derived
  int n_tiles = 0;
  int n_long = 0;
  int n_chunks = 0;
  Tile *tiles = nullptr;          // device
  LongRow *longs = nullptr;       // device
  double *chunk_part = nullptr;   // device, n_chunks
  unsigned *long_cnt = nullptr;   // device, n_long (zero between launches)
  double *long_dot = nullptr;     // device, 2 * n_long
  int spmv_grid[5] = {0, 0, 0, 0, 0}; // CTAs of the SpMV launch, per kernel variant
  int variant = 0;                // SpMV kernel variant in use
  int short_max = kShortRow;      // rows up to this length: one thread, in row order
  int longest_row = 0;
  // cached derived data
  void *inv_diag = nullptr;       // 1/diag(A), dtype elements
  bool inv_diag_valid = false;
  void *extras = nullptr;         // precision/format variants (mixed solver)
  void *transpose = nullptr;      // cached A^T for the transposed SpMV
  void *sor = nullptr;            // the SOR solver's sweep (mlsh_krylov.cu)
  // 16-bit column format (FP32 plans made for the mixed solver)
  uint16_t *col16 = nullptr;      // device, nnz: col - tile_base[tile]
  int *tile_base = nullptr;       // device, n_tiles
  // offset-slot layout (FP32 plans made for the mixed solver), or null
  SlotFormat *slots = nullptr;
};

// ------------------------------------------------------------ launches ---
// Launch kernel `k` as a programmatic dependent of the stream's previous
// kernel: its CTAs may start while that kernel's last CTAs retire, and the
// kernel waits (griddepcontrol.wait, first thing) until the previous one has
// completed and its writes are visible.  Only kernels that make that wait
// before touching global memory may be launched this way.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*k)(KArgs...), int grid, int block, size_t smem,
                                    cudaStream_t s, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, static_cast<Args &&>(args)...);
}

// -------------------------------------------------------------- errors ---
void set_last_error(const char *where, cudaError_t e);

#define MLSH_CUDA_TRY(expr)                         \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) {                        \
      ::mlsh::set_last_error(#expr, _e);            \
      return MLSH_ERR_CUDA;                         \
    }                                               \
  } while (0)

// Plan- and handle-owned buffers come from the stream-ordered pool of the
// stream that uses them: no device-wide synchronization on allocation or
// release, so plans can be built and destroyed while kernels of other
// streams (a persistent serving kernel, say) keep running.
template <typename P>
inline cudaError_t pool_alloc(P **ptr, size_t bytes, cudaStream_t s) {
  return cudaMallocAsync(reinterpret_cast<void **>(ptr), bytes, s);
}
inline void pool_free(void *ptr, cudaStream_t s) {
  if (ptr) cudaFreeAsync(ptr, s);
}

inline int dtype_size(int dtype) {
  return dtype == MLSH_F64 ? 8 : (dtype == MLSH_F32 ? 4 : 0);
}

}  // namespace mlsh

struct mlsh_handle_s {
  mlsh::Handle h;
};
struct mlsh_csr_plan_s {
  mlsh::CsrPlan p;
};
