"""Python harness over the C ABI (used by the tests and the benchmark).

Device memory comes from torch (plumbing only); every computation is a call
into libmlsh.so through ctypes.  Names follow the reference's vocabulary:
a ``Crs`` is a device-resident ``matrix::CRS<T>`` after ``send()``, ``matvec``
is ``blas::matvec``, ``cg_solve``/``bicgstab_solve`` are
``equation::CG``/``BiCGSTAB`` ``::solve``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _dtype_code(np_dtype) -> int:
    if np.dtype(np_dtype) == np.float64:
        return _abi.F64
    if np.dtype(np_dtype) == np.float32:
        return _abi.F32
    raise TypeError(f"unsupported dtype {np_dtype}")


def _torch_dtype(np_dtype):
    return torch.float64 if np.dtype(np_dtype) == np.float64 else torch.float32


def ptr(t) -> int:
    return t.data_ptr() if t is not None else 0


class Handle:
    """mlsh_handle bound to the current torch CUDA stream."""

    def __init__(self, stream=None):
        self.lib = _abi.load()
        h = C.c_void_p()
        _abi.check(self.lib.mlsh_create(C.byref(h)), "mlsh_create")
        self.h = h
        if stream is None and torch is not None and torch.cuda.is_available():
            stream = torch.cuda.current_stream().cuda_stream
        if stream:
            _abi.check(self.lib.mlsh_set_stream(self.h, C.c_void_p(stream)), "set_stream")

    def close(self):
        if self.h:
            self.lib.mlsh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        return _abi.check(self.lib.mlsh_synchronize(self.h), "synchronize")

    # ---------------------------------------------------------- vector BLAS
    def dot(self, x, y) -> float:
        out = C.c_double()
        _abi.check(self.lib.mlsh_dot(self.h, _dtype_code(_np(x)), x.numel(), ptr(x), ptr(y),
                                     C.byref(out)), "dot")
        return out.value

    def nrm2(self, x) -> float:
        out = C.c_double()
        _abi.check(self.lib.mlsh_nrm2(self.h, _dtype_code(_np(x)), x.numel(), ptr(x),
                                      C.byref(out)), "nrm2")
        return out.value

    def axpy(self, alpha, x, y):
        _abi.check(self.lib.mlsh_axpy(self.h, _dtype_code(_np(x)), x.numel(), alpha, ptr(x),
                                      ptr(y)), "axpy")

    def xpay(self, alpha, x, y):
        _abi.check(self.lib.mlsh_xpay(self.h, _dtype_code(_np(x)), x.numel(), alpha, ptr(x),
                                      ptr(y)), "xpay")

    def axpyz(self, alpha, x, y, z):
        _abi.check(self.lib.mlsh_axpyz(self.h, _dtype_code(_np(x)), x.numel(), alpha, ptr(x),
                                       ptr(y), ptr(z)), "axpyz")

    def copy(self, x, y):
        _abi.check(self.lib.mlsh_copy(self.h, _dtype_code(_np(x)), x.numel(), ptr(x), ptr(y)),
                   "copy")

    def vsub(self, a, b, y):
        _abi.check(self.lib.mlsh_vsub(self.h, _dtype_code(_np(a)), a.numel(), ptr(a), ptr(b),
                                      ptr(y)), "vsub")

    def vmul(self, a, b, y):
        _abi.check(self.lib.mlsh_vmul(self.h, _dtype_code(_np(a)), a.numel(), ptr(a), ptr(b),
                                      ptr(y)), "vmul")

    def vreciprocal(self, a, y):
        _abi.check(self.lib.mlsh_vreciprocal(self.h, _dtype_code(_np(a)), a.numel(), ptr(a),
                                             ptr(y)), "vreciprocal")


def _np(t):
    return np.float64 if t.dtype == torch.float64 else np.float32


class Crs:
    """A CRS matrix resident on the device, with its SpMV plan."""

    def __init__(self, handle: Handle, n_rows, n_cols, row_ptr, col_ind, val,
                 validate=True):
        self.handle = handle
        self.lib = handle.lib
        self.n_rows, self.n_cols = int(n_rows), int(n_cols)
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.dtype = np.dtype(val.dtype)
        self.nnz = int(rp[-1]) if len(rp) else 0
        dev = torch.device("cuda")
        self.d_rp = torch.from_numpy(rp).to(dev)
        self.d_ci = torch.from_numpy(np.ascontiguousarray(col_ind, dtype=np.int32)).to(dev)
        self.d_val = torch.from_numpy(np.ascontiguousarray(val)).to(dev)
        plan = C.c_void_p()
        _abi.check(self.lib.mlsh_csr_plan_create(
            handle.h, self.n_rows, self.n_cols, self.nnz, ptr(self.d_rp), ptr(self.d_ci),
            ptr(self.d_val), _dtype_code(self.dtype), rp.ctypes.data_as(C.c_void_p),
            1 if validate else 0, C.byref(plan)), "csr_plan_create")
        self.plan = plan

    def close(self):
        # after its handle is destroyed the plan's memory went with it
        if self.plan and self.handle.h:
            self.lib.mlsh_csr_plan_destroy(self.plan)
        self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        nt, nl, b = C.c_int(), C.c_int(), C.c_int64()
        _abi.check(self.lib.mlsh_csr_plan_info(self.plan, C.byref(nt), C.byref(nl),
                                               C.byref(b)), "plan_info")
        return {"n_tiles": nt.value, "n_long_rows": nl.value, "spmv_bytes": b.value}

    def autotune(self, x, y):
        """Time every SpMV kernel variant on this matrix; keep the fastest."""
        v, sec = C.c_int(), C.c_double()
        _abi.check(self.lib.mlsh_csr_plan_autotune(self.handle.h, self.plan, ptr(x), ptr(y),
                                                   C.byref(v), C.byref(sec)), "autotune")
        return v.value, sec.value

    def set_variant(self, v):
        _abi.check(self.lib.mlsh_csr_plan_set_variant(self.plan, int(v)), "set_variant")

    def set_short_rows(self, max_len):
        _abi.check(self.lib.mlsh_csr_plan_set_short_rows(self.plan, int(max_len)),
                   "set_short_rows")

    def tuning(self):
        """(kernel variant, short-row limit) in use."""
        v, sm = C.c_int(), C.c_int()
        _abi.check(self.lib.mlsh_csr_plan_tuning(self.plan, C.byref(v), C.byref(sm)), "tuning")
        return v.value, sm.value

    def set_layout(self, layout) -> bool:
        """0: CRS, 1: offset-slot layout (FP32 plans); True if it is in use."""
        applied = C.c_int()
        _abi.check(self.lib.mlsh_csr_plan_set_layout(self.plan, int(layout), C.byref(applied)),
                   "set_layout")
        return bool(applied.value)

    def variant(self):
        v, nv = C.c_int(), C.c_int()
        _abi.check(self.lib.mlsh_csr_plan_get_variant(self.plan, C.byref(v), C.byref(nv)),
                   "get_variant")
        return v.value, nv.value

    def matvec(self, x, y, alpha=1.0, beta=0.0):
        _abi.check(self.lib.mlsh_spmv(self.handle.h, self.plan, alpha, ptr(x), beta, ptr(y)),
                   "spmv")

    def diag(self, out):
        _abi.check(self.lib.mlsh_csr_diag(self.handle.h, self.plan, ptr(out)), "diag")

    def matvec_t(self, x, y, alpha=1.0, beta=0.0):
        """y = alpha A^T x + beta y (blas::matvec_T)."""
        _abi.check(self.lib.mlsh_spmv_transpose(self.handle.h, self.plan, alpha, ptr(x), beta,
                                                ptr(y)), "spmv_transpose")

    def values_changed(self):
        _abi.check(self.lib.mlsh_csr_plan_values_changed(self.plan), "values_changed")


def coo_sort(handle: Handle, n_rows, n_cols, d_row, d_col, d_val, merge=True):
    """Sort device COO tensors in place by (row, col); returns the entry
    count (after merging duplicates when `merge`)."""
    k = C.c_int64()
    _abi.check(handle.lib.mlsh_coo_sort(
        handle.h, int(n_rows), int(n_cols), int(d_row.numel()), ptr(d_row), ptr(d_col),
        ptr(d_val), _dtype_code(np.dtype(str(d_val.dtype).replace("torch.", ""))), int(merge),
        C.byref(k)), "coo_sort")
    return k.value


def coo_to_csr(handle: Handle, n_rows, d_row, nnz=None):
    """Row pointer (device int32 tensor) of a row-sorted device COO."""
    nnz = int(d_row.numel()) if nnz is None else int(nnz)
    rp = torch.empty(n_rows + 1, dtype=torch.int32, device=d_row.device)
    _abi.check(handle.lib.mlsh_coo_to_csr(handle.h, int(n_rows), nnz, ptr(d_row), ptr(rp)),
               "coo_to_csr")
    return rp


def csr_transpose(handle: Handle, n_rows, n_cols, d_rp, d_ci, d_val):
    """(rp_t, ci_t, val_t) device tensors of A^T."""
    nnz = int(d_ci.numel())
    rp_t = torch.empty(n_cols + 1, dtype=torch.int32, device=d_rp.device)
    ci_t = torch.empty(max(nnz, 1), dtype=torch.int32, device=d_rp.device)
    v_t = torch.empty(max(nnz, 1), dtype=d_val.dtype, device=d_rp.device)
    _abi.check(handle.lib.mlsh_csr_transpose(
        handle.h, int(n_rows), int(n_cols), nnz, ptr(d_rp), ptr(d_ci), ptr(d_val),
        _dtype_code(np.dtype(str(d_val.dtype).replace("torch.", ""))), ptr(rp_t), ptr(ci_t),
        ptr(v_t)), "csr_transpose")
    return rp_t, ci_t[:nnz], v_t[:nnz]


@dataclass
class SolveResult:
    status: int
    iters: int
    resid: float
    outer: int = 0


def _opts(tol, maxiter, miniter, precond, use_graph, check_every, engine, cluster_rows,
          time_limit=0.0, wait_polls=0):
    o = _abi.SolverOpts()
    _abi.load().mlsh_solver_opts_default(C.byref(o))
    o.tol, o.maxiter, o.miniter = tol, maxiter, miniter
    o.precond = precond
    o.use_graph = 1 if use_graph else 0
    o.check_every = check_every
    o.engine = engine
    o.cluster_rows = cluster_rows
    o.time_limit = float(time_limit)
    o.wait_polls = int(wait_polls)
    return o


def _solve(fn, A: Crs, b, x, tol, maxiter, miniter=0, precond=_abi.PRECOND_JACOBI,
           use_graph=True, check_every=0, engine=_abi.ENGINE_AUTO, cluster_rows=0,
           history=None, time_limit=0.0):
    o = _opts(tol, maxiter, miniter, precond, use_graph, check_every, engine, cluster_rows,
              time_limit=time_limit)
    if history is not None:
        o.history = history.ctypes.data_as(C.POINTER(C.c_double))
        o.history_len = len(history)
    r = _abi.SolverResult()
    st = fn(A.handle.h, A.plan, ptr(b), ptr(x), C.byref(o), C.byref(r))
    if st not in (_abi.SUCCESS, _abi.SOLVER_MAXITER, _abi.SOLVER_BREAKDOWN,
                  _abi.SOLVER_RESIDUAL_NAN, _abi.SOLVER_SIZE_ERROR):
        raise _abi.MlshError(st, "solve")
    return SolveResult(st, int(r.iters), float(r.final_resid), int(r.outer_iters))


def _solve_mixed(fn, A: Crs, b, x, tol, maxiter, inner_tol=1e-4, miniter=0,
                 precond=_abi.PRECOND_JACOBI, engine=_abi.ENGINE_AUTO, history=None,
                 use_graph=True):
    o = _opts(tol, maxiter, miniter, precond, use_graph, 0, engine, 0)
    if history is not None:
        o.history = history.ctypes.data_as(C.POINTER(C.c_double))
        o.history_len = len(history)
    r = _abi.SolverResult()
    st = fn(A.handle.h, A.plan, ptr(b), ptr(x), C.byref(o), inner_tol, C.byref(r))
    if st not in (_abi.SUCCESS, _abi.SOLVER_MAXITER, _abi.SOLVER_BREAKDOWN,
                  _abi.SOLVER_RESIDUAL_NAN, _abi.SOLVER_SIZE_ERROR):
        raise _abi.MlshError(st, "mixed solve")
    return SolveResult(st, int(r.iters), float(r.final_resid), int(r.outer_iters))


def cg_solve_mixed(A: Crs, b, x, tol, maxiter, **kw) -> SolveResult:
    """FP32 inner CG inside FP64 iterative refinement (A must be FP64)."""
    return _solve_mixed(A.lib.mlsh_cg_solve_mixed, A, b, x, tol, maxiter, **kw)


def bicgstab_solve_mixed(A: Crs, b, x, tol, maxiter, **kw) -> SolveResult:
    """FP32 inner BiCGSTAB inside FP64 iterative refinement (A must be FP64)."""
    return _solve_mixed(A.lib.mlsh_bicgstab_solve_mixed, A, b, x, tol, maxiter, **kw)


class Batch:
    """Independent systems stored as one concatenated CRS (column indices
    local to each system), solved together by mlsh_batch_solve."""

    def __init__(self, handle: Handle, systems, dtype=np.float64):
        self.handle = handle
        self.lib = handle.lib
        self.dtype = np.dtype(dtype)
        sizes = np.array([len(rp) - 1 for rp, _, _ in systems], np.int64)
        self.row_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        nnz = np.array([int(rp[-1]) for rp, _, _ in systems], np.int64)
        nnz_off = np.concatenate([[0], np.cumsum(nnz)])
        total_rows = int(self.row_off[-1])
        rp_all = np.empty(total_rows + 1, np.int64)
        for k, (rp, _, _) in enumerate(systems):
            rp_all[self.row_off[k]:self.row_off[k + 1]] = rp[:-1] + nnz_off[k]
        rp_all[-1] = nnz_off[-1]
        if nnz_off[-1] > 2**31 - 1:
            raise ValueError("concatenated nnz exceeds int32")
        ci_all = np.concatenate([ci for _, ci, _ in systems]).astype(np.int32)
        v_all = np.concatenate([v for _, _, v in systems]).astype(self.dtype)
        dev = torch.device("cuda")
        self.d_rp = torch.from_numpy(rp_all.astype(np.int32)).to(dev)
        self.d_ci = torch.from_numpy(ci_all).to(dev)
        self.d_val = torch.from_numpy(v_all).to(dev)
        self.n_systems = len(systems)
        bh = C.c_void_p()
        _abi.check(self.lib.mlsh_batch_create(
            handle.h, self.n_systems, self.row_off.ctypes.data_as(C.c_void_p), ptr(self.d_rp),
            ptr(self.d_ci), ptr(self.d_val), _dtype_code(self.dtype), C.byref(bh)),
            "batch_create")
        self.b = bh

    def close(self):
        if self.b and self.handle.h:
            self.lib.mlsh_batch_destroy(self.b)
        self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, kind, d_b, d_x, tol, maxiter, miniter=0, precond=_abi.PRECOND_JACOBI,
              time_limit=0.0):
        """kind 'cg' or 'bicgstab'; tol: scalar or per-system absolute array."""
        o = _opts(1e-8, maxiter, miniter, precond, True, 0, _abi.ENGINE_CLUSTER, 0,
                  time_limit=time_limit)
        tol_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(tol, np.float64),
                                                       (self.n_systems,)))
        status = np.zeros(self.n_systems, np.int32)
        iters = np.zeros(self.n_systems, np.int64)
        resid = np.zeros(self.n_systems, np.float64)
        st = self.lib.mlsh_batch_solve(
            self.handle.h, self.b, 0 if kind == "cg" else 1, ptr(d_b), ptr(d_x),
            tol_arr.ctypes.data_as(C.c_void_p), C.byref(o), status.ctypes.data_as(C.c_void_p),
            iters.ctypes.data_as(C.c_void_p), resid.ctypes.data_as(C.c_void_p))
        if st < _abi.NOT_IMPL:
            raise _abi.MlshError(st, "batch_solve")
        return status, iters, resid

    def solve_mixed(self, d_b, d_x, tol, maxiter, inner_tol=1e-2, miniter=0,
                    precond=_abi.PRECOND_JACOBI):
        """Jacobi-CG on every system, FP32 iterations with FP64 refreshes."""
        o = _opts(1e-8, maxiter, miniter, precond, True, 0, _abi.ENGINE_CLUSTER, 0)
        tol_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(tol, np.float64),
                                                       (self.n_systems,)))
        status = np.zeros(self.n_systems, np.int32)
        iters = np.zeros(self.n_systems, np.int64)
        resid = np.zeros(self.n_systems, np.float64)
        st = self.lib.mlsh_batch_cg_solve_mixed(
            self.handle.h, self.b, ptr(d_b), ptr(d_x), tol_arr.ctypes.data_as(C.c_void_p),
            C.byref(o), float(inner_tol), status.ctypes.data_as(C.c_void_p),
            iters.ctypes.data_as(C.c_void_p), resid.ctypes.data_as(C.c_void_p))
        if st < _abi.NOT_IMPL:
            raise _abi.MlshError(st, "batch_cg_solve_mixed")
        return status, iters, resid

    def autotune(self, kind, d_b, d_x, tol, maxiter, precond=_abi.PRECOND_JACOBI,
                 inner_tol=1e-2):
        """Times one batched solve per rows-per-CTA cap (1,024 to 16,384) and
        keeps the fastest for later solves of `kind` ('cg', 'bicgstab' or
        'mixed'); d_x comes back as it went in.  Returns (cap, seconds of the
        fastest solve)."""
        o = _opts(1e-8, maxiter, 0, precond, True, 0, _abi.ENGINE_CLUSTER, 0)
        tol_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(tol, np.float64),
                                                       (self.n_systems,)))
        cap, secs = C.c_int(0), C.c_double(0.0)
        _abi.check(self.lib.mlsh_batch_autotune(
            self.handle.h, self.b, {"cg": 0, "bicgstab": 1, "mixed": 2}[kind], ptr(d_b),
            ptr(d_x), tol_arr.ctypes.data_as(C.c_void_p), C.byref(o), float(inner_tol),
            C.byref(cap), C.byref(secs)), "batch_autotune")
        return cap.value, secs.value

    def info(self, kind):
        """(rows-per-CTA cap, number of groups) for 'cg', 'bicgstab' or 'mixed'."""
        cap, n_groups = C.c_int(0), C.c_int(0)
        _abi.check(self.lib.mlsh_batch_info(self.b, {"cg": 0, "bicgstab": 1, "mixed": 2}[kind],
                                            C.byref(cap), C.byref(n_groups)), "batch_info")
        return cap.value, n_groups.value


def cg_solve(A: Crs, b, x, tol, maxiter, **kw) -> SolveResult:
    return _solve(A.lib.mlsh_cg_solve, A, b, x, tol, maxiter, **kw)


def bicgstab_solve(A: Crs, b, x, tol, maxiter, **kw) -> SolveResult:
    return _solve(A.lib.mlsh_bicgstab_solve, A, b, x, tol, maxiter, **kw)


class Precond:
    """mlsh_precond: SOR / IC(0) / ILU(0) of a plan's matrix
    (equation::SOR / IC / ILU create_precond; apply = apply_precond)."""

    def __init__(self, A: Crs, kind, omega=1.9):
        self.A = A
        self.lib = A.lib
        self.kind = int(kind)
        h = C.c_void_p()
        _abi.check(self.lib.mlsh_precond_create(A.handle.h, A.plan, self.kind, float(omega),
                                                C.byref(h)), "mlsh_precond_create")
        self.pc = h

    def zero_pivot(self):
        """(row, structural): the first zero pivot, row -1 if none."""
        row, structural = C.c_int64(), C.c_int()
        _abi.check(self.lib.mlsh_precond_zero_pivot(self.pc, C.byref(row), C.byref(structural)))
        return int(row.value), int(structural.value)

    def apply(self, r, z):
        _abi.check(self.lib.mlsh_precond_apply(self.A.handle.h, self.pc, ptr(r), ptr(z)),
                   "mlsh_precond_apply")

    def info(self):
        """(levels of the lower sweep, levels of the upper sweep, blocks)."""
        lo, up, nb = C.c_int(), C.c_int(), C.c_int64()
        _abi.check(self.lib.mlsh_precond_info(self.pc, C.byref(lo), C.byref(up), C.byref(nb)))
        return int(lo.value), int(up.value), int(nb.value)

    def sweep_form(self):
        """Kernel form of the (lower, upper) sweep: 0 flags across the GPU,
        1 single CTA, 2 single CTA with the record ring; -1 none."""
        lo, up = C.c_int(), C.c_int()
        _abi.check(self.lib.mlsh_precond_sweep_form(self.pc, C.byref(lo), C.byref(up)))
        return int(lo.value), int(up.value)

    def factor(self):
        """SOR: M (n); IC / ILU: the factor's values in A's pattern (nnz)."""
        n = self.A.n_rows if self.kind == _abi.PRECOND_SOR else self.A.nnz
        out = torch.empty(max(n, 1), dtype=_torch_dtype(self.A.dtype), device="cuda")
        _abi.check(self.lib.mlsh_precond_factor(self.A.handle.h, self.pc, ptr(out)))
        return out[:n]

    def close(self):
        if self.pc and self.A.handle.h:
            self.lib.mlsh_precond_destroy(self.pc)
        self.pc = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _solve_pc(fn, A: Crs, pc: Precond, b, x, tol, maxiter, miniter=0, use_graph=True,
              check_every=0, history=None, wait_polls=0):
    o = _opts(tol, maxiter, miniter, _abi.PRECOND_NONE, use_graph, check_every,
              _abi.ENGINE_KERNELS, 0, wait_polls=wait_polls)
    if history is not None:
        o.history = history.ctypes.data_as(C.POINTER(C.c_double))
        o.history_len = len(history)
    r = _abi.SolverResult()
    st = fn(A.handle.h, A.plan, pc.pc, ptr(b), ptr(x), C.byref(o), C.byref(r))
    if st not in (_abi.SUCCESS, _abi.SOLVER_MAXITER, _abi.SOLVER_BREAKDOWN,
                  _abi.SOLVER_RESIDUAL_NAN, _abi.SOLVER_SIZE_ERROR):
        raise _abi.MlshError(st, "preconditioned solve")
    return SolveResult(st, int(r.iters), float(r.final_resid), 0)


def cg_solve_precond(A: Crs, pc: Precond, b, x, tol, maxiter, **kw) -> SolveResult:
    """CG preconditioned by an SOR / IC / ILU object."""
    return _solve_pc(A.lib.mlsh_cg_solve_precond, A, pc, b, x, tol, maxiter, **kw)


def bicgstab_solve_precond(A: Crs, pc: Precond, b, x, tol, maxiter, **kw) -> SolveResult:
    """BiCGSTAB preconditioned by an SOR / IC / ILU object."""
    return _solve_pc(A.lib.mlsh_bicgstab_solve_precond, A, pc, b, x, tol, maxiter, **kw)


def sor_solve(A: Crs, b, x, tol, maxiter, omega=1.9, miniter=0, use_graph=True,
              check_every=0, history=None) -> SolveResult:
    """equation::SOR::solve: relative stopping rule ||r|| / ||b|| < tol."""
    o = _opts(tol, maxiter, miniter, _abi.PRECOND_NONE, use_graph, check_every,
              _abi.ENGINE_KERNELS, 0)
    if history is not None:
        o.history = history.ctypes.data_as(C.POINTER(C.c_double))
        o.history_len = len(history)
    r = _abi.SolverResult()
    st = A.lib.mlsh_sor_solve(A.handle.h, A.plan, ptr(b), ptr(x), float(omega), C.byref(o),
                              C.byref(r))
    if st not in (_abi.SUCCESS, _abi.SOLVER_MAXITER, _abi.SOLVER_BREAKDOWN,
                  _abi.SOLVER_RESIDUAL_NAN, _abi.SOLVER_SIZE_ERROR):
        raise _abi.MlshError(st, "SOR solve")
    return SolveResult(st, int(r.iters), float(r.final_resid), 0)


@dataclass
class ServeResult:
    status: int
    path: int          # 0 cluster ring, 1 worker lane
    iters: int
    resid: float
    t_submit: float
    t_admit: float
    t_done: float
    x: np.ndarray


class Server:
    """Solve server over mlsh_server_*: requests (host CRS + right-hand
    side) are submitted while others run and come back with their
    solution and timestamps on the server's clock."""

    def __init__(self, memory_budget=8 << 30, n_lanes=2):
        self.lib = _abi.load()
        s = C.c_void_p()
        _abi.check(self.lib.mlsh_server_create(int(memory_budget), int(n_lanes), C.byref(s)),
                   "server_create")
        self.s = s
        self._live = {}  # request id -> host arrays kept alive until done

    def submit(self, kind, row_ptr, col_ind, val, b, tol, maxiter, x0=None,
               precond=_abi.PRECOND_JACOBI, precision="fp64", inner_tol=1e-4) -> int:
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_ind, np.int32)
        v = np.ascontiguousarray(val, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        n = len(rp) - 1
        xo = np.zeros(n, np.float64)
        r = _abi.Request()
        r.kind = 0 if kind == "cg" else 1
        r.precision = 0 if precision == "fp64" else 1
        r.precond = precond
        r.n = n
        r.nnz = int(rp[-1])
        r.row_ptr = rp.ctypes.data
        r.col_ind = ci.ctypes.data if len(ci) else None
        r.val = v.ctypes.data if len(v) else None
        r.b = bb.ctypes.data if n else None
        r.x0 = None if x0a is None else x0a.ctypes.data
        r.x_out = xo.ctypes.data if n else None
        r.tol = float(tol)
        r.maxiter = int(maxiter)
        r.inner_tol = float(inner_tol)
        rid = C.c_int64()
        _abi.check(self.lib.mlsh_server_submit(self.s, C.byref(r), C.byref(rid)), "server_submit")
        self._live[rid.value] = (rp, ci, v, bb, x0a, xo)
        return rid.value

    def _result(self, rid, res):
        arrays = self._live.pop(rid)
        return ServeResult(res.status, res.path, res.iters, res.resid, res.t_submit,
                           res.t_admit, res.t_done, arrays[5])

    def poll(self, rid):
        """The result if request `rid` has finished, else None."""
        res = _abi.RequestResult()
        st = self.lib.mlsh_server_poll(self.s, rid, C.byref(res))
        if st == _abi.PENDING:
            return None
        _abi.check(st, "server_poll")
        return self._result(rid, res)

    def wait(self, rid) -> ServeResult:
        res = _abi.RequestResult()
        _abi.check(self.lib.mlsh_server_wait(self.s, rid, C.byref(res)), "server_wait")
        return self._result(rid, res)

    def drain(self):
        _abi.check(self.lib.mlsh_server_drain(self.s), "server_drain")

    def now(self) -> float:
        return self.lib.mlsh_server_now(self.s)

    def stats(self):
        """(serving-kernel launches, lane solves) since creation."""
        a, b = C.c_int64(), C.c_int64()
        _abi.check(self.lib.mlsh_server_stats(self.s, C.byref(a), C.byref(b)), "server_stats")
        return a.value, b.value

    def close(self):
        if self.s:
            self.lib.mlsh_server_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
