// Mixed-precision solves: FP32 inner Krylov iterations inside an FP64
// iterative-refinement loop (include/mlsh.h: mlsh_*_solve_mixed).
//
//   repeat
//     r = b - A x                 FP64 SpMV on the FP64 values, fused ||r||
//     stop when ||r|| < tol       (the true residual, not a recurrence)
//     s = ||r||;  r32 = r / s     rounded to FP32
//     A32 d = r32                 CG / BiCGSTAB in FP32 on an FP32 copy of the
//                                 values (in the offset-slot layout, or with
//                                 16-bit column offsets, when the structure
//                                 allows: mlsh_slots.cu), to inner tolerance
//                                 (relative; ||r32|| = 1); dots and norms are
//                                 still accumulated in FP64
//     x += s * d                  FP64 update
//
// The inner iterations read 6-8 bytes per nonzero instead of 12 and half
// the vector bytes, which is where the speed-up over the plain FP64 solve
// comes from; the FP64 residual keeps the answer exact to the outer
// tolerance.  The FP32 copy is derived once per plan and dropped when the
// plan's values change.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "mlsh_cluster.cuh"
#include "mlsh_core.cuh"

namespace mlsh {

struct MixedExtras {
  mlsh_csr_plan plan32 = nullptr;  // FP32 plan over val32 (same structure)
  float *val32 = nullptr;
  double *r64 = nullptr;
  float *r32 = nullptr;
  float *d32 = nullptr;
  bool valid = false;
  int scaled = 0;  // val32 holds A D^-1 (Jacobi folded in) rather than A
};

namespace {

struct ToF32Body : NoPrep {
  const double *src;
  float *dst;
  double scale;
  __device__ void operator()(int64_t i, double *) const { dst[i] = (float)(src[i] * scale); }
};

struct AddScaledBody : NoPrep {  // x += s * d (FP64)
  double *x;
  const float *d;
  double s;
  __device__ void operator()(int64_t i, double *) const { x[i] = s * (double)d[i] + x[i]; }
};

// val32[j] = val[j] / A(col[j], col[j]): A D^-1 rounded once to FP32.
__global__ void to_f32_right_scaled(const double *val, const int *col, const double *dinv,
                                    int64_t nnz, float *out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz;
       j += (int64_t)gridDim.x * blockDim.x)
    out[j] = (float)(val[j] * dinv[col[j]]);
}

// The FP32 values of the extras in the requested form.
int fill_val32(Handle &h, CsrPlan &p, MixedExtras *m, const double *dinv) {
  if (p.nnz <= 0) return MLSH_SUCCESS;
  if (dinv) {
    const int64_t nnz = p.nnz;
    const unsigned g = (unsigned)std::min<int64_t>((nnz + 255) / 256, (int64_t)h.num_sms * 16);
    to_f32_right_scaled<<<g, 256, 0, h.stream>>>(static_cast<const double *>(p.val), p.col_ind,
                                                 dinv, nnz, m->val32);
    MLSH_CUDA_TRY(cudaGetLastError());
    return MLSH_SUCCESS;
  }
  ToF32Body cv;
  cv.src = static_cast<const double *>(p.val);
  cv.dst = m->val32;
  cv.scale = 1.0;
  RedArgs ra{h.partials, h.counters, nullptr};
  vec_kernel<0, false, ToF32Body>
      <<<vec_grid(p.nnz, h.num_sms), kVecThreads, 0, h.stream>>>(p.nnz, cv, ra);
  MLSH_CUDA_TRY(cudaGetLastError());
  return MLSH_SUCCESS;
}

template <typename Body>
int run_plain(const Handle &h, int64_t n, const Body &b) {
  RedArgs ra{h.partials, h.counters, nullptr};
  vec_kernel<0, false, Body><<<vec_grid(n, h.num_sms), kVecThreads, 0, h.stream>>>(n, b, ra);
  MLSH_CUDA_TRY(cudaGetLastError());
  return MLSH_SUCCESS;
}

// Per-tile min/max column (one CTA per tile).
__global__ void tile_col_range(const Tile *tiles, const int *col, int *tmin, int *tmax) {
  const Tile t = tiles[blockIdx.x];
  int lo = INT32_MAX, hi = INT32_MIN;
  for (int j = t.nnz_begin + threadIdx.x; j < t.nnz_end; j += blockDim.x) {
    const int c = col[j];
    lo = min(lo, c);
    hi = max(hi, c);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ int slo[32], shi[32];
  if ((threadIdx.x & 31) == 0) {
    slo[threadIdx.x >> 5] = lo;
    shi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      lo = min(lo, slo[w]);
      hi = max(hi, shi[w]);
    }
    tmin[blockIdx.x] = lo;
    tmax[blockIdx.x] = hi;
  }
}

__global__ void tile_col16(const Tile *tiles, const int *col, const int *base, uint16_t *out) {
  const Tile t = tiles[blockIdx.x];
  const int b = base[blockIdx.x];
  for (int j = t.nnz_begin + threadIdx.x; j < t.nnz_end; j += blockDim.x)
    out[j] = (uint16_t)(col[j] - b);
}

// 16-bit column offsets for the FP32 plan when every tile's columns span
// fewer than 65,536 values; otherwise the plan keeps 32-bit columns.
int build_col16(CsrPlan &q, cudaStream_t s) {
  if (q.n_tiles == 0 || q.nnz == 0) return MLSH_SUCCESS;
  int *tmin = nullptr, *tmax = nullptr;
  MLSH_CUDA_TRY(pool_alloc(&tmin, sizeof(int) * q.n_tiles, s));
  MLSH_CUDA_TRY(pool_alloc(&tmax, sizeof(int) * q.n_tiles, s));
  tile_col_range<<<q.n_tiles, 256, 0, s>>>(q.tiles, q.col_ind, tmin, tmax);
  std::vector<int> lo(q.n_tiles), hi(q.n_tiles);
  cudaMemcpyAsync(lo.data(), tmin, sizeof(int) * q.n_tiles, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(hi.data(), tmax, sizeof(int) * q.n_tiles, cudaMemcpyDeviceToHost, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  pool_free(tmax, s);
  if (e != cudaSuccess) {
    pool_free(tmin, s);
    set_last_error("tile column ranges", e);
    return MLSH_ERR_CUDA;
  }
  for (int t = 0; t < q.n_tiles; ++t) {
    if (lo[t] > hi[t]) lo[t] = 0;  // empty tile
    if ((int64_t)hi[t] - lo[t] >= 65536) {
      pool_free(tmin, s);
      return MLSH_SUCCESS;  // not compressible: keep 32-bit columns
    }
  }
  cudaMemcpyAsync(tmin, lo.data(), sizeof(int) * q.n_tiles, cudaMemcpyHostToDevice, s);
  uint16_t *c16 = nullptr;
  if (pool_alloc(&c16, sizeof(uint16_t) * (size_t)q.nnz, s) != cudaSuccess) {
    cudaGetLastError();
    pool_free(tmin, s);
    return MLSH_SUCCESS;  // no room: keep 32-bit columns
  }
  tile_col16<<<q.n_tiles, 256, 0, s>>>(q.tiles, q.col_ind, tmin, c16);
  MLSH_CUDA_TRY(cudaGetLastError());
  q.col16 = c16;
  q.tile_base = tmin;
  return MLSH_SUCCESS;
}

void free_extras(MixedExtras *m, cudaStream_t s) {
  if (!m) return;
  if (m->plan32) mlsh_csr_plan_destroy(m->plan32);
  cudaStreamSynchronize(s);
  for (void *d : {(void *)m->val32, (void *)m->r64, (void *)m->r32, (void *)m->d32})
    pool_free(d, s);
  m->plan32 = nullptr;
  m->val32 = nullptr;
  m->r64 = nullptr;
  m->r32 = nullptr;
  m->d32 = nullptr;
  m->valid = false;
}

// The FP32 copy of p: plain (dinv == nullptr) or right-scaled by the FP64
// inverse diagonal `dinv`.  Switching between the two rewrites the values
// only; the structure (tiles, 16-bit columns) is kept.
int ensure_extras(mlsh_handle hs, CsrPlan &p, MixedExtras **out, const double *dinv) {
  Handle &h = hs->h;
  MixedExtras *m = static_cast<MixedExtras *>(p.extras);
  if (!m) {
    m = new (std::nothrow) MixedExtras();
    if (!m) return MLSH_ERR_OOM;
    p.extras = m;
  }
  const int want = dinv != nullptr ? 1 : 0;
  if (m->valid) {
    if (m->scaled != want) {
      int st = fill_val32(h, p, m, dinv);
      if (st != MLSH_SUCCESS) return st;
      mlsh_csr_plan_values_changed(m->plan32);
      st = slots_build(m->plan32->p, h.stream);
      if (st != MLSH_SUCCESS) return st;
      m->scaled = want;
    }
    *out = m;
    return MLSH_SUCCESS;
  }
  free_extras(m, h.stream);
  const size_t n = (size_t)std::max(p.n_rows, 1);
  const size_t nnz = (size_t)std::max(p.nnz, 1);
  if (pool_alloc(&m->val32, sizeof(float) * nnz, h.stream) != cudaSuccess ||
      pool_alloc(&m->r64, sizeof(double) * n, h.stream) != cudaSuccess ||
      pool_alloc(&m->r32, sizeof(float) * n, h.stream) != cudaSuccess ||
      pool_alloc(&m->d32, sizeof(float) * n, h.stream) != cudaSuccess) {
    cudaGetLastError();
    free_extras(m, h.stream);
    return MLSH_ERR_OOM;
  }
  {
    const int st = fill_val32(h, p, m, dinv);
    if (st != MLSH_SUCCESS) return st;
  }
  m->scaled = want;
  int st = mlsh_csr_plan_create(hs, p.n_rows, p.n_cols, p.nnz, p.row_ptr, p.col_ind, m->val32,
                                MLSH_F32, nullptr, 0, &m->plan32);
  if (st != MLSH_SUCCESS) return st;
  CsrPlan &q = m->plan32->p;
  q.variant = p.variant;
  // the offset-slot layout where the structure allows, else 16-bit columns
  st = slots_build(q, h.stream);
  if (st != MLSH_SUCCESS) return st;
  if (q.slots == nullptr) {
    st = build_col16(q, h.stream);
    if (st != MLSH_SUCCESS) return st;
  }
  m->valid = true;
  *out = m;
  return MLSH_SUCCESS;
}

}  // namespace

void mixed_release(CsrPlan &p) {
  MixedExtras *m = static_cast<MixedExtras *>(p.extras);
  if (m) {
    free_extras(m, p.handle ? p.handle->stream : nullptr);
    delete m;
    p.extras = nullptr;
  }
}

void mixed_invalidate(CsrPlan &p) {
  MixedExtras *m = static_cast<MixedExtras *>(p.extras);
  if (m && m->plan32) {
    // values changed: the FP32 copy is rebuilt at the next mixed solve
    free_extras(m, p.handle ? p.handle->stream : nullptr);
  }
}

int mixed_solve(int kind, mlsh_handle hs, mlsh_csr_plan ps, const void *d_b, void *d_x,
                const mlsh_solver_opts *opts, double inner_tol, mlsh_solver_result *res) {
  if (!hs || !ps || !opts || !(inner_tol > 0.0) || !(inner_tol < 1.0))
    return MLSH_ERR_INVALID_ARG;
  Handle &h = hs->h;
  CsrPlan &p = ps->p;
  if (p.dtype != MLSH_F64) return MLSH_ERR_INVALID_ARG;
  if (p.n_rows != p.n_cols) {
    if (res) res->status = MLSH_SOLVER_SIZE_ERROR;
    return MLSH_SOLVER_SIZE_ERROR;
  }
  mlsh_solver_result local{};
  if (!res) res = &local;
  const int64_t n = p.n_rows;
  if (n == 0) return kind == 0 ? mlsh_cg_solve(hs, ps, d_b, d_x, opts, res)
                               : mlsh_bicgstab_solve(hs, ps, d_b, d_x, opts, res);
  if (!d_b || !d_x) return MLSH_ERR_INVALID_ARG;
  // Large systems (the FP32 iteration on the kernel engine): BiCGSTAB with
  // reliable updates in one graph.  Systems that fit a thread-block cluster
  // keep the restarted refinement below, whose inner solves run on it.
  const bool inner_on_cluster =
      opts->engine == MLSH_ENGINE_CLUSTER ||
      (opts->engine == MLSH_ENGINE_AUTO && opts->maxiter <= kClusterMaxIterAuto &&
       cluster_rows_for(kind, MLSH_F32, n, opts->cluster_rows) != 0);
  MixedExtras *m = nullptr;
  if (kind == 1 && !inner_on_cluster) {
    if (opts->precond != MLSH_PRECOND_NONE && opts->precond != MLSH_PRECOND_JACOBI)
      return MLSH_ERR_INVALID_ARG;
    const void *dinv = nullptr;
    if (opts->precond == MLSH_PRECOND_JACOBI) {
      const int s2 = plan_inv_diag(p, h.stream, &dinv);
      if (s2 != MLSH_SUCCESS) return s2;
    }
    int s1 = ensure_extras(hs, p, &m, static_cast<const double *>(dinv));
    if (s1 != MLSH_SUCCESS) return s1;
    return mixed_bicgstab_kernels(h, p, m->plan32->p, m->r64,
                                  static_cast<const double *>(dinv), d_b, d_x, opts, inner_tol,
                                  res);
  }
  int st = ensure_extras(hs, p, &m, nullptr);
  if (st != MLSH_SUCCESS) return st;

  mlsh_solver_opts in = *opts;
  in.tol = inner_tol;
  in.miniter = 0;
  in.history = nullptr;
  in.history_len = 0;
  const bool want_hist = opts->history != nullptr && opts->history_len > 0;
  int64_t inner_total = 0;
  int outer = 0;
  double resid = 0.0;
  int status = kRunning;
  constexpr int kMaxOuter = 100;
  while (true) {
    // r = b - A x in FP64, fused ||r||^2 into scalars[0]
    cudaError_t e = launch_spmv_t<double, kDotSelf, kDotNone>(
        p, h, -1.0, static_cast<const double *>(d_x), 1.0, static_cast<const double *>(d_b),
        m->r64, nullptr, nullptr, h.scalars, nullptr, h.stream);
    if (e != cudaSuccess) {
      set_last_error("mixed: residual", e);
      return MLSH_ERR_CUDA;
    }
    MLSH_CUDA_TRY(cudaMemcpyAsync(h.host_scalars, h.scalars, sizeof(double),
                                  cudaMemcpyDeviceToHost, h.stream));
    MLSH_CUDA_TRY(cudaStreamSynchronize(h.stream));
    resid = std::sqrt(h.host_scalars[0]);
    if (want_hist && outer < opts->history_len) opts->history[outer] = resid;
    if (resid < opts->tol && opts->miniter <= inner_total) {
      status = MLSH_SUCCESS;
      break;
    }
    if (std::isnan(resid)) {
      status = MLSH_SOLVER_RESIDUAL_NAN;
      break;
    }
    if (inner_total >= opts->maxiter || outer >= kMaxOuter) {
      status = MLSH_SOLVER_MAXITER;
      break;
    }
    // r32 = r / ||r||, d32 = 0, inner solve A32 d32 = r32
    ToF32Body cv;
    cv.src = m->r64;
    cv.dst = m->r32;
    cv.scale = 1.0 / resid;
    st = run_plain(h, n, cv);
    if (st != MLSH_SUCCESS) return st;
    MLSH_CUDA_TRY(cudaMemsetAsync(m->d32, 0, sizeof(float) * (size_t)n, h.stream));
    in.maxiter = opts->maxiter - inner_total;
    mlsh_solver_result ir{};
    st = kind == 0 ? mlsh_cg_solve(hs, m->plan32, m->r32, m->d32, &in, &ir)
                   : mlsh_bicgstab_solve(hs, m->plan32, m->r32, m->d32, &in, &ir);
    if (st < MLSH_NOT_IMPL) return st;  // library error
    inner_total += ir.iters;
    ++outer;
    if (ir.status == MLSH_SOLVER_RESIDUAL_NAN) {
      status = MLSH_SOLVER_RESIDUAL_NAN;
      break;
    }
    // x += s * d (the partial correction of a breakdown is still applied)
    AddScaledBody up;
    up.x = static_cast<double *>(d_x);
    up.d = m->d32;
    up.s = resid;
    st = run_plain(h, n, up);
    if (st != MLSH_SUCCESS) return st;
    if (ir.status == MLSH_SOLVER_BREAKDOWN && ir.iters == 0) {
      status = MLSH_SOLVER_BREAKDOWN;
      break;
    }
  }
  res->status = status;
  res->iters = inner_total;
  res->final_resid = resid;
  res->outer_iters = outer;
  return status;
}

}  // namespace mlsh

using namespace mlsh;

extern "C" {

int mlsh_cg_solve_mixed(mlsh_handle hs, mlsh_csr_plan ps, const void *d_b, void *d_x,
                        const mlsh_solver_opts *opts, double inner_tol,
                        mlsh_solver_result *result) {
  return mixed_solve(0, hs, ps, d_b, d_x, opts, inner_tol, result);
}

static void storage_of(const CsrPlan &p, int *layout, int64_t *bytes) {
  if (p.slots) {
    *layout = MLSH_LAYOUT_SLOTS;
    *bytes = p.slots->bytes();
    return;
  }
  *layout = MLSH_LAYOUT_CRS;
  const int64_t V = dtype_size(p.dtype);
  const int64_t C = p.col16 ? 2 : 4;
  *bytes = (int64_t)p.nnz * (V + C) + ((int64_t)p.n_rows + 1) * 4 +
           (p.col16 ? (int64_t)p.n_tiles * 4 : 0);
}

int mlsh_csr_plan_storage(mlsh_csr_plan ps, int which, int *layout, int64_t *matrix_bytes) {
  if (!ps || (which != 0 && which != 1)) return MLSH_ERR_INVALID_ARG;
  int lay = -1;
  int64_t b = 0;
  if (which == 0) {
    storage_of(ps->p, &lay, &b);
  } else {
    const MixedExtras *m = static_cast<const MixedExtras *>(ps->p.extras);
    if (m && m->valid && m->plan32) storage_of(m->plan32->p, &lay, &b);
  }
  if (layout) *layout = lay;
  if (matrix_bytes) *matrix_bytes = b;
  return MLSH_SUCCESS;
}

int mlsh_bicgstab_solve_mixed(mlsh_handle hs, mlsh_csr_plan ps, const void *d_b, void *d_x,
                              const mlsh_solver_opts *opts, double inner_tol,
                              mlsh_solver_result *result) {
  return mixed_solve(1, hs, ps, d_b, d_x, opts, inner_tol, result);
}

}  // extern "C"
