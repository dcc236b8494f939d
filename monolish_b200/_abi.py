"""ctypes declarations for the C ABI in include/mlsh.h.

The library is loaded from this package's ``lib/`` directory; a missing
library raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libmlsh.so")

SUCCESS = 0
SOLVER_SIZE_ERROR = -1
SOLVER_MAXITER = -2
SOLVER_BREAKDOWN = -3
SOLVER_RESIDUAL_NAN = -4
NOT_IMPL = -10
ERR_CUDA = -20
ERR_INVALID_ARG = -21
ERR_INVALID_CSR = -22
ERR_OOM = -23
ERR_TIMEOUT = -24
ERR_NO_DEVICE = -25
PENDING = 1

F64 = 0
F32 = 1
PRECOND_NONE = 0
PRECOND_JACOBI = 1
PRECOND_SOR = 2
PRECOND_IC = 3
PRECOND_ILU = 4

vp = C.c_void_p
i32 = C.c_int
i64 = C.c_int64
f64 = C.c_double


class SolverOpts(C.Structure):
    _fields_ = [("tol", f64), ("maxiter", i64), ("miniter", i64), ("precond", i32),
                ("use_graph", i32), ("check_every", i32), ("engine", i32),
                ("history", C.POINTER(f64)), ("history_len", i64),
                ("cluster_rows", i32), ("reserved", i32), ("time_limit", f64),
                ("wait_polls", i64)]


ENGINE_AUTO = 0
ENGINE_KERNELS = 1
ENGINE_CLUSTER = 2


class SolverResult(C.Structure):
    _fields_ = [("status", i32), ("outer_iters", i32), ("iters", i64), ("final_resid", f64)]


class Request(C.Structure):
    _fields_ = [("kind", i32), ("precision", i32), ("precond", i32), ("n", i32), ("nnz", i32),
                ("reserved", i32), ("row_ptr", vp), ("col_ind", vp), ("val", vp), ("b", vp),
                ("x0", vp), ("x_out", vp), ("tol", f64), ("maxiter", i64), ("inner_tol", f64)]


class RequestResult(C.Structure):
    _fields_ = [("status", i32), ("path", i32), ("iters", i64), ("resid", f64),
                ("t_submit", f64), ("t_admit", f64), ("t_done", f64)]


# name -> (restype, argtypes); every symbol include/mlsh.h declares
SIGNATURES = {
    "mlsh_version": (i32, []),
    "mlsh_status_string": (C.c_char_p, [i32]),
    "mlsh_last_error": (C.c_char_p, []),
    "mlsh_create": (i32, [C.POINTER(vp)]),
    "mlsh_destroy": (i32, [vp]),
    "mlsh_set_stream": (i32, [vp, vp]),
    "mlsh_get_stream": (i32, [vp, C.POINTER(vp)]),
    "mlsh_synchronize": (i32, [vp]),
    "mlsh_device_alloc": (i32, [C.c_size_t, C.POINTER(vp)]),
    "mlsh_device_free": (i32, [vp]),
    "mlsh_memcpy_h2d": (i32, [vp, vp, vp, C.c_size_t]),
    "mlsh_memcpy_d2h": (i32, [vp, vp, vp, C.c_size_t]),
    "mlsh_memcpy_d2d": (i32, [vp, vp, vp, C.c_size_t]),
    "mlsh_memcpy_h2d_async": (i32, [vp, vp, vp, C.c_size_t]),
    "mlsh_memcpy_d2h_async": (i32, [vp, vp, vp, C.c_size_t]),
    "mlsh_csr_plan_create": (i32, [vp, i32, i32, i32, vp, vp, vp, i32, vp, i32, C.POINTER(vp)]),
    "mlsh_csr_plan_destroy": (i32, [vp]),
    "mlsh_csr_plan_values_changed": (i32, [vp]),
    "mlsh_csr_plan_info": (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i64)]),
    "mlsh_csr_plan_autotune": (i32, [vp, vp, vp, vp, C.POINTER(i32), C.POINTER(f64)]),
    "mlsh_csr_plan_set_variant": (i32, [vp, i32]),
    "mlsh_csr_plan_get_variant": (i32, [vp, C.POINTER(i32), C.POINTER(i32)]),
    "mlsh_csr_plan_set_layout": (i32, [vp, i32, C.POINTER(i32)]),
    "mlsh_csr_plan_set_short_rows": (i32, [vp, i32]),
    "mlsh_csr_plan_tuning": (i32, [vp, C.POINTER(i32), C.POINTER(i32)]),
    "mlsh_csr_plan_storage": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i64)]),
    "mlsh_spmv": (i32, [vp, vp, f64, vp, f64, vp]),
    "mlsh_csr_diag": (i32, [vp, vp, vp]),
    "mlsh_spmv_transpose": (i32, [vp, vp, f64, vp, f64, vp]),
    "mlsh_coo_sort": (i32, [vp, i32, i32, i64, vp, vp, vp, i32, i32, C.POINTER(i64)]),
    "mlsh_coo_to_csr": (i32, [vp, i32, i64, vp, vp]),
    "mlsh_csr_transpose": (i32, [vp, i32, i32, i32, vp, vp, vp, i32, vp, vp, vp]),
    "mlsh_dot": (i32, [vp, i32, i64, vp, vp, C.POINTER(f64)]),
    "mlsh_nrm2": (i32, [vp, i32, i64, vp, C.POINTER(f64)]),
    "mlsh_dot_device": (i32, [vp, i32, i64, vp, vp, vp]),
    "mlsh_nrm2_device": (i32, [vp, i32, i64, vp, vp]),
    "mlsh_dot_noalloc": (i32, [i32, i64, vp, vp, vp, vp]),
    "mlsh_axpy": (i32, [vp, i32, i64, f64, vp, vp]),
    "mlsh_xpay": (i32, [vp, i32, i64, f64, vp, vp]),
    "mlsh_axpyz": (i32, [vp, i32, i64, f64, vp, vp, vp]),
    "mlsh_copy": (i32, [vp, i32, i64, vp, vp]),
    "mlsh_vsub": (i32, [vp, i32, i64, vp, vp, vp]),
    "mlsh_vmul": (i32, [vp, i32, i64, vp, vp, vp]),
    "mlsh_vreciprocal": (i32, [vp, i32, i64, vp, vp]),
    "mlsh_fill": (i32, [vp, i32, i64, f64, vp]),
    "mlsh_solver_opts_default": (i32, [C.POINTER(SolverOpts)]),
    "mlsh_cg_solve": (i32, [vp, vp, vp, vp, C.POINTER(SolverOpts), C.POINTER(SolverResult)]),
    "mlsh_bicgstab_solve": (i32, [vp, vp, vp, vp, C.POINTER(SolverOpts),
                                  C.POINTER(SolverResult)]),
    "mlsh_cg_solve_mixed": (i32, [vp, vp, vp, vp, C.POINTER(SolverOpts), f64,
                                  C.POINTER(SolverResult)]),
    "mlsh_bicgstab_solve_mixed": (i32, [vp, vp, vp, vp, C.POINTER(SolverOpts), f64,
                                        C.POINTER(SolverResult)]),
    "mlsh_precond_create": (i32, [vp, vp, i32, f64, C.POINTER(vp)]),
    "mlsh_precond_zero_pivot": (i32, [vp, C.POINTER(i64), C.POINTER(i32)]),
    "mlsh_precond_apply": (i32, [vp, vp, vp, vp]),
    "mlsh_precond_factor": (i32, [vp, vp, vp]),
    "mlsh_precond_destroy": (i32, [vp]),
    "mlsh_precond_info": (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i64)]),
    "mlsh_precond_sweep_form": (i32, [vp, C.POINTER(i32), C.POINTER(i32)]),
    "mlsh_cg_solve_precond": (i32, [vp, vp, vp, vp, vp, C.POINTER(SolverOpts),
                                    C.POINTER(SolverResult)]),
    "mlsh_bicgstab_solve_precond": (i32, [vp, vp, vp, vp, vp, C.POINTER(SolverOpts),
                                          C.POINTER(SolverResult)]),
    "mlsh_sor_solve": (i32, [vp, vp, vp, vp, f64, C.POINTER(SolverOpts),
                             C.POINTER(SolverResult)]),
    "mlsh_batch_create": (i32, [vp, i32, vp, vp, vp, vp, i32, C.POINTER(vp)]),
    "mlsh_batch_destroy": (i32, [vp]),
    "mlsh_batch_solve": (i32, [vp, vp, i32, vp, vp, vp, C.POINTER(SolverOpts), vp, vp, vp]),
    "mlsh_batch_autotune": (i32, [vp, vp, i32, vp, vp, vp, C.POINTER(SolverOpts), f64,
                                  C.POINTER(i32), C.POINTER(f64)]),
    "mlsh_batch_info": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32)]),
    "mlsh_batch_cg_solve_mixed": (i32, [vp, vp, vp, vp, vp, C.POINTER(SolverOpts), f64, vp, vp,
                                        vp]),
    "mlsh_server_create": (i32, [C.c_size_t, i32, C.POINTER(vp)]),
    "mlsh_server_submit": (i32, [vp, C.POINTER(Request), C.POINTER(i64)]),
    "mlsh_server_poll": (i32, [vp, i64, C.POINTER(RequestResult)]),
    "mlsh_server_wait": (i32, [vp, i64, C.POINTER(RequestResult)]),
    "mlsh_server_drain": (i32, [vp]),
    "mlsh_server_now": (f64, [vp]),
    "mlsh_server_stats": (i32, [vp, C.POINTER(i64), C.POINTER(i64)]),
    "mlsh_server_destroy": (i32, [vp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libmlsh.so (raises OSError if it is missing or fails to load)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"CUDA library not built: {path} (run __graft_entry__.build())")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MlshError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        lib = _lib
        msg = lib.mlsh_status_string(status).decode() if lib else str(status)
        detail = lib.mlsh_last_error().decode() if lib else ""
        super().__init__(f"{what}: {msg} ({status}) {detail}".strip())
        self.status = status


def check(status: int, what: str = "", ok=(SUCCESS,)):
    if status not in ok:
        raise MlshError(status, what)
    return status
