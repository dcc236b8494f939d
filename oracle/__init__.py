"""Checker bindings (TEST INFRASTRUCTURE ONLY).

Two CPU implementations of the reference's solve path:

* ``Restatement`` -- ``_build/libmlsh_oracle.so``, the C restatement in
  mlsh_oracle.c (always buildable);
* ``Reference``   -- ``_ref/libmlsh_refcapi.so``, the reference monolish CPU
  library compiled from the reference sources (oracle/Makefile), called
  through its own public API.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg may use
this package; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_LIB = os.path.join(HERE, "_build", "libmlsh_oracle.so")
REFERENCE_LIB = os.path.join(HERE, "_ref", "libmlsh_refcapi.so")

P = C.c_void_p


def _p(a):
    return a.ctypes.data_as(P)


class _Base:
    def _solve_args(self, rp, ci, v, b, x):
        return (len(rp) - 1, _p(rp), _p(ci), _p(v), _p(b), _p(x))


class Restatement:
    def __init__(self, path=RESTATEMENT_LIB):
        if not os.path.exists(path):
            raise OSError(f"oracle restatement not built: {path}")
        self.lib = lib = C.CDLL(path)
        I, L, D = C.c_int, C.c_long, C.c_double
        for nm in ("oracle_spmv_d", "oracle_spmv_s"):
            getattr(lib, nm).argtypes = [I, P, P, P, P, P]
        lib.oracle_spmv_ab_d.argtypes = [I, P, P, P, D, P, D, P]
        for nm in ("oracle_spmv_t_d", "oracle_spmv_t_s"):
            getattr(lib, nm).argtypes = [I, I, P, P, P, P, P]
        lib.oracle_coo_sort_d.argtypes = [L, P, P, P, I]
        lib.oracle_coo_sort_d.restype = L
        lib.oracle_coo_rowptr.argtypes = [I, L, P, P]
        lib.oracle_csr_transpose_d.argtypes = [I, I, P, P, P, P, P, P]
        lib.oracle_dot_d.argtypes = [L, P, P]
        lib.oracle_dot_d.restype = D
        lib.oracle_nrm2_d.argtypes = [L, P]
        lib.oracle_nrm2_d.restype = D
        lib.oracle_true_relres_d.argtypes = [I, P, P, P, P, P]
        lib.oracle_true_relres_d.restype = D
        for nm in ("oracle_cg_d", "oracle_cg_s", "oracle_bicgstab_d", "oracle_bicgstab_s"):
            f = getattr(lib, nm)
            f.argtypes = [I, P, P, P, P, P, D, L, L, I, D, C.POINTER(L), C.POINTER(D)]
            f.restype = I
        for sfx in ("d", "s"):
            f = getattr(lib, f"oracle_precond_factor_{sfx}")
            f.argtypes = [I, P, P, P, I, D, P, C.POINTER(L)]
            f.restype = I
            f = getattr(lib, f"oracle_precond_apply_{sfx}")
            f.argtypes = [I, P, P, P, I, D, P, P]
            f.restype = I
            f = getattr(lib, f"oracle_sor_{sfx}")
            f.argtypes = [I, P, P, P, P, P, D, D, L, L, P, C.POINTER(L), C.POINTER(D)]
            f.restype = I

    def spmv(self, rp, ci, v, x):
        n = len(rp) - 1
        y = np.zeros(n, v.dtype)
        fn = self.lib.oracle_spmv_d if v.dtype == np.float64 else self.lib.oracle_spmv_s
        fn(n, _p(rp), _p(ci), _p(v), _p(x), _p(y))
        return y

    def spmv_ab(self, rp, ci, v, alpha, x, beta, y):
        y = y.copy()
        self.lib.oracle_spmv_ab_d(len(rp) - 1, _p(rp), _p(ci), _p(v), alpha, _p(x), beta, _p(y))
        return y

    def spmv_t(self, rp, ci, v, x, n_cols):
        """y = A^T x (the reference's serial row loop)."""
        y = np.zeros(n_cols, v.dtype)
        fn = self.lib.oracle_spmv_t_d if v.dtype == np.float64 else self.lib.oracle_spmv_t_s
        fn(len(rp) - 1, n_cols, _p(rp), _p(ci), _p(v), _p(x), _p(y))
        return y

    def coo_sort(self, row, col, val, merge):
        r = np.array(row, np.int32)
        c = np.array(col, np.int32)
        v = np.array(val, np.float64)
        k = self.lib.oracle_coo_sort_d(len(r), _p(r), _p(c), _p(v), int(merge))
        return r[:k].copy(), c[:k].copy(), v[:k].copy()

    def coo_rowptr(self, n_rows, row):
        row = np.ascontiguousarray(row, np.int32)
        rp = np.zeros(n_rows + 1, np.int32)
        self.lib.oracle_coo_rowptr(n_rows, len(row), _p(row), _p(rp))
        return rp

    def csr_transpose(self, rp, ci, v, n_cols):
        nnz = int(rp[-1])
        rp_t = np.zeros(n_cols + 1, np.int32)
        ci_t = np.zeros(nnz, np.int32)
        v_t = np.zeros(nnz, np.float64)
        self.lib.oracle_csr_transpose_d(len(rp) - 1, n_cols, _p(rp), _p(ci), _p(v), _p(rp_t),
                                        _p(ci_t), _p(v_t))
        return rp_t, ci_t, v_t

    def dot(self, x, y):
        return self.lib.oracle_dot_d(len(x), _p(x), _p(y))

    def nrm2(self, x):
        return self.lib.oracle_nrm2_d(len(x), _p(x))

    def true_relres(self, rp, ci, v, b, x):
        return self.lib.oracle_true_relres_d(len(rp) - 1, _p(rp), _p(ci), _p(v), _p(b), _p(x))

    def _solve(self, name, rp, ci, v, b, x0, tol, maxiter, miniter=0, precond=1, omega=1.9):
        """precond: 0 none, 1 Jacobi, 2 SOR (omega), 3 IC(0), 4 ILU(0)."""
        sfx = "d" if v.dtype == np.float64 else "s"
        x = x0.copy()
        it, res = C.c_long(), C.c_double()
        st = getattr(self.lib, f"oracle_{name}_{sfx}")(
            len(rp) - 1, _p(rp), _p(ci), _p(v), _p(b), _p(x), tol, maxiter, miniter, precond,
            omega, C.byref(it), C.byref(res))
        return st, it.value, res.value, x

    def precond_factor(self, rp, ci, v, kind, omega=1.9):
        """(values, pivot): SOR M (n), IC / ILU the factor in A's pattern."""
        sfx = "d" if v.dtype == np.float64 else "s"
        n = len(rp) - 1
        out = np.zeros(n if kind == 2 else int(rp[-1]), v.dtype)
        piv = C.c_long()
        st = getattr(self.lib, f"oracle_precond_factor_{sfx}")(
            n, _p(rp), _p(ci), _p(v), kind, omega, _p(out), C.byref(piv))
        if st != 0:
            raise ValueError("rows not sorted")
        return out, piv.value

    def precond_apply(self, rp, ci, v, kind, r, omega=1.9):
        sfx = "d" if v.dtype == np.float64 else "s"
        z = np.zeros_like(r)
        getattr(self.lib, f"oracle_precond_apply_{sfx}")(
            len(rp) - 1, _p(rp), _p(ci), _p(v), kind, omega, _p(r), _p(z))
        return z

    def sor(self, rp, ci, v, b, x0, tol, maxiter, omega=1.9, miniter=0, history=False):
        """(status, iters, final resid, x[, relative residual history])."""
        sfx = "d" if v.dtype == np.float64 else "s"
        x = x0.copy()
        it, res = C.c_long(), C.c_double()
        hist = np.zeros(max(int(maxiter), 1), np.float64) if history else None
        st = getattr(self.lib, f"oracle_sor_{sfx}")(
            len(rp) - 1, _p(rp), _p(ci), _p(v), _p(b), _p(x), omega, tol, maxiter, miniter,
            _p(hist) if history else None, C.byref(it), C.byref(res))
        if history:
            return st, it.value, res.value, x, hist[:it.value].copy()
        return st, it.value, res.value, x

    def cg(self, *a, **k):
        return self._solve("cg", *a, **k)

    def bicgstab(self, *a, **k):
        return self._solve("bicgstab", *a, **k)


class Reference:
    """The reference CPU library, built from its own sources."""

    def __init__(self, path=REFERENCE_LIB):
        if not os.path.exists(path):
            raise OSError(f"reference CPU build not present: {path}")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        # read by the OpenMP runtime when the library loads
        os.environ.setdefault("OMP_PROC_BIND", "close")
        self.lib = lib = C.CDLL(path)
        I, L, D = C.c_int, C.c_long, C.c_double
        lib.ref_max_threads.restype = I
        lib.ref_set_threads.argtypes = [I]
        for nm in ("ref_spmv_d", "ref_spmv_s"):
            f = getattr(lib, nm)
            f.argtypes = [I, I, P, P, P, P, P, I, P]
            f.restype = I
        for nm in ("ref_cg_d", "ref_cg_s", "ref_bicgstab_d", "ref_bicgstab_s"):
            f = getattr(lib, nm)
            f.argtypes = [I, I, P, P, P, P, P, D, L, I, C.POINTER(L), C.POINTER(D), C.POINTER(D)]
            f.restype = I
        lib.ref_dot_d.argtypes = [L, P, P]
        lib.ref_dot_d.restype = D
        lib.ref_nrm2_d.argtypes = [L, P]
        lib.ref_nrm2_d.restype = D
        lib.ref_axpy_d.argtypes = [L, D, P, P]
        lib.ref_xpay_d.argtypes = [L, D, P, P]
        lib.ref_axpyz_d.argtypes = [L, D, P, P, P]
        lib.ref_random_vector_d.argtypes = [L, D, D, C.c_uint, P]
        lib.ref_laplacian_2d5p_d.argtypes = [I, I, P, P, P]
        lib.ref_laplacian_2d5p_d.restype = L
        lib.ref_spmv_t_d.argtypes = [I, I, I, P, P, P, P, P]
        lib.ref_spmv_t_d.restype = I
        lib.ref_coo_sort_d.argtypes = [I, I, L, P, P, P, I]
        lib.ref_coo_sort_d.restype = L
        lib.ref_coo_to_crs_d.argtypes = [I, I, L, P, P, P, P]
        lib.ref_coo_to_crs_d.restype = I
        for sfx in ("d", "s"):
            f = getattr(lib, f"ref_sor_{sfx}")
            f.argtypes = [I, I, P, P, P, P, P, D, D, L, C.POINTER(L), C.POINTER(D), C.POINTER(D)]
            f.restype = I
            f = getattr(lib, f"ref_sor_apply_{sfx}")
            f.argtypes = [I, I, P, P, P, D, P, P]
            f.restype = I

    def threads(self):
        return self.lib.ref_max_threads()

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def spmv(self, rp, ci, v, x, reps=1):
        n = len(rp) - 1
        y = np.zeros(n, v.dtype)
        sec = np.zeros(2)
        fn = self.lib.ref_spmv_d if v.dtype == np.float64 else self.lib.ref_spmv_s
        fn(n, int(rp[-1]), _p(rp), _p(ci), _p(v), _p(x), _p(y), reps, _p(sec))
        return y, float(sec[0]), float(sec[1])

    def spmv_t(self, rp, ci, v, x, n_cols):
        y = np.zeros(n_cols, np.float64)
        self.lib.ref_spmv_t_d(len(rp) - 1, n_cols, int(rp[-1]), _p(rp), _p(ci), _p(v), _p(x),
                              _p(y))
        return y

    def coo_sort(self, n_rows, n_cols, row, col, val, merge):
        r = np.array(row, np.int32)
        c = np.array(col, np.int32)
        v = np.array(val, np.float64)
        k = self.lib.ref_coo_sort_d(n_rows, n_cols, len(r), _p(r), _p(c), _p(v), int(merge))
        return r[:k].copy(), c[:k].copy(), v[:k].copy()

    def coo_rowptr(self, n_rows, n_cols, row, col, val):
        row = np.ascontiguousarray(row, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        rp = np.zeros(n_rows + 1, np.int32)
        self.lib.ref_coo_to_crs_d(n_rows, n_cols, len(row), _p(row), _p(col), _p(val), _p(rp))
        return rp

    def _solve(self, name, rp, ci, v, b, x0, tol, maxiter, precond=1):
        sfx = "d" if v.dtype == np.float64 else "s"
        x = x0.copy()
        it, res, sec = C.c_long(), C.c_double(), C.c_double()
        st = getattr(self.lib, f"ref_{name}_{sfx}")(
            len(rp) - 1, int(rp[-1]), _p(rp), _p(ci), _p(v), _p(b), _p(x), tol, maxiter,
            precond, C.byref(it), C.byref(res), C.byref(sec))
        return st, it.value, res.value, x, sec.value

    def cg(self, *a, **k):
        """precond: 0 none, 1 Jacobi, 2 SOR (omega 1.9)."""
        return self._solve("cg", *a, **k)

    def bicgstab(self, *a, **k):
        return self._solve("bicgstab", *a, **k)

    def sor(self, rp, ci, v, b, x0, tol, maxiter, omega=1.9):
        """equation::SOR::solve: (status, iters, final resid, x, seconds)."""
        sfx = "d" if v.dtype == np.float64 else "s"
        x = x0.copy()
        it, res, sec = C.c_long(), C.c_double(), C.c_double()
        st = getattr(self.lib, f"ref_sor_{sfx}")(
            len(rp) - 1, int(rp[-1]), _p(rp), _p(ci), _p(v), _p(b), _p(x), omega, tol,
            maxiter, C.byref(it), C.byref(res), C.byref(sec))
        return st, it.value, res.value, x, sec.value

    def sor_apply(self, rp, ci, v, r, omega=1.9):
        """equation::SOR create_precond + apply_precond: z = M^{-1} r."""
        sfx = "d" if v.dtype == np.float64 else "s"
        z = np.zeros_like(r)
        getattr(self.lib, f"ref_sor_apply_{sfx}")(len(rp) - 1, int(rp[-1]), _p(rp), _p(ci),
                                                  _p(v), omega, _p(r), _p(z))
        return z

    def dot(self, x, y):
        return self.lib.ref_dot_d(len(x), _p(x), _p(y))

    def nrm2(self, x):
        return self.lib.ref_nrm2_d(len(x), _p(x))

    def axpy(self, a, x, y):
        y = y.copy()
        self.lib.ref_axpy_d(len(x), a, _p(x), _p(y))
        return y

    def xpay(self, a, x, y):
        y = y.copy()
        self.lib.ref_xpay_d(len(x), a, _p(x), _p(y))
        return y

    def axpyz(self, a, x, y):
        z = np.zeros_like(x)
        self.lib.ref_axpyz_d(len(x), a, _p(x), _p(y), _p(z))
        return z

    def random_vector(self, n, lo, hi, seed):
        out = np.zeros(n)
        self.lib.ref_random_vector_d(n, lo, hi, seed, _p(out))
        return out

    def laplacian_2d5p(self, m, n):
        nn = m * n
        nnz = self.lib.ref_laplacian_2d5p_d(m, n, None, None, None)
        rp = np.zeros(nn + 1, np.int32)
        ci = np.zeros(nnz, np.int32)
        v = np.zeros(nnz)
        self.lib.ref_laplacian_2d5p_d(m, n, _p(rp), _p(ci), _p(v))
        return nn, rp, ci, v


def restatement():
    return Restatement()


def reference_or_none():
    try:
        return Reference()
    except OSError:
        return None
