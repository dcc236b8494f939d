"""CRS SpMV on the GPU against the oracle (through the C ABI).

Tolerance: rows of up to 8 nonzeros (every row of the stencil workloads)
are summed by one thread in the reference's order (products rounded, then
added in row order), so they must be bit-identical to the CPU row loop.
Longer rows are summed as 8-entry segments / CTA-wide chunks;
for them |y - y_ref|_i <= 4 * len_i * eps * (|A||x|)_i (the standard
summation error bound), which is below 1e-14 relative for the workloads'
row lengths.
"""
import os

import numpy as np
import pytest

from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def run_spmv(handle, n_rows, n_cols, rp, ci, v, x, alpha=1.0, beta=0.0, y0=None):
    import torch
    from monolish_b200.device import Crs
    A = Crs(handle, n_rows, n_cols, rp, ci, v)
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dy = (torch.from_numpy(np.ascontiguousarray(y0)).cuda() if y0 is not None
          else torch.full((n_rows,), float("nan"), dtype=dx.dtype, device="cuda"))
    A.matvec(dx, dy, alpha, beta)
    handle.sync()
    out = dy.cpu().numpy()
    A.close()
    return out


def check(rp, ci, v, x, y, y_ref):
    lens = np.diff(rp)
    short = lens <= 8
    assert np.array_equal(y[short], y_ref[short]), "short rows must match bitwise"
    if (~short).any():
        absax = np.zeros(len(lens))
        np.add.at(absax, np.repeat(np.arange(len(lens)), lens), np.abs(v * x[ci]))
        eps = np.finfo(v.dtype).eps
        bound = 4 * lens * eps * absax
        err = np.abs(y.astype(np.float64) - y_ref.astype(np.float64))
        assert (err[~short] <= bound[~short]).all()


def test_golden_zipf_long_rows(handle, restatement):
    g = np.load(os.path.join(GOLDEN, "zipf_spmv.npz"))
    rp, ci, v, x = g["rp"], g["ci"], g["v"], g["x"]
    n = len(rp) - 1
    assert np.diff(rp).max() > 1792  # exercises chunked long rows
    y = run_spmv(handle, n, n, rp, ci, v, x)
    check(rp, ci, v, x, y, g["y"])
    ys = run_spmv(handle, n, n, rp, ci, v.astype(np.float32), x.astype(np.float32))
    check(rp, ci, v.astype(np.float32), x.astype(np.float32), ys, g["y_s"])


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_poisson2d_bitwise(handle, restatement, dt):
    n, rp, ci, v = W.poisson2d(128)
    x = W.uniform_mt(n, -1, 1, 1).astype(dt)
    v = v.astype(dt)
    y = run_spmv(handle, n, n, rp, ci, v, x)
    assert np.array_equal(y, restatement.spmv(rp, ci, v, x))


def test_poisson3d_bitwise(handle, restatement):
    n, rp, ci, v = W.poisson3d(40)
    x = W.uniform_mt(n, -1, 1, 1)
    y = run_spmv(handle, n, n, rp, ci, v, x)
    assert np.array_equal(y, restatement.spmv(rp, ci, v, x))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_zipf_random(handle, restatement, dt):
    n, rp, ci, v = W.zipf(60000, seed=1, maxlen=10000)
    x = W.uniform_mt(n, -1, 1, 1).astype(dt)
    v = v.astype(dt)
    y = run_spmv(handle, n, n, rp, ci, v, x)
    check(rp, ci, v, x, y, restatement.spmv(rp, ci, v, x))


def test_alpha_beta(handle, restatement):
    n, rp, ci, v = W.zipf(5000, seed=4, maxlen=5000)
    x = W.uniform_mt(n, -1, 1, 2)
    y0 = W.uniform_mt(n, -1, 1, 3)
    y = run_spmv(handle, n, n, rp, ci, v, x, alpha=-0.5, beta=2.0, y0=y0)
    ref = restatement.spmv_ab(rp, ci, v, -0.5, x, 2.0, y0)
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13)
    # beta = 0 must not read y (y0 full of NaN)
    y = run_spmv(handle, n, n, rp, ci, v, x, alpha=1.0, beta=0.0,
                 y0=np.full(n, np.nan))
    assert np.isfinite(y).all()


def test_edge_shapes(handle, restatement):
    rng = np.random.default_rng(5)
    # empty rows, a single huge row, rectangular, n = 1
    lens = rng.integers(0, 4, 3000)
    lens[::7] = 0
    lens[1500] = 20000
    n_cols = 25000
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n_cols, L, replace=False)) for L in lens]).astype(
        np.int32)
    v = rng.uniform(-1, 1, rp[-1])
    x = rng.uniform(-1, 1, n_cols)
    y = run_spmv(handle, len(lens), n_cols, rp, ci, v, x)
    ref = restatement.spmv(rp, ci, v, x)
    check(rp, ci, v, x, y, ref)
    assert (y[lens == 0] == 0).all()
    # one row, one column
    y = run_spmv(handle, 1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                 np.array([3.0]), np.array([2.0]))
    assert y[0] == 6.0


def test_unaligned_arrays(handle, restatement):
    """Value/column arrays starting off a 16-byte boundary (ragged TMA ends)."""
    import torch
    from monolish_b200.device import Crs
    n, rp, ci, v = W.zipf(4000, seed=9, maxlen=3000)
    x = W.uniform_mt(n, -1, 1, 4)
    ref = restatement.spmv(rp, ci, v, x)
    for off in (1, 3):
        A = Crs(handle, n, n, rp, ci, v)
        big_v = torch.zeros(len(v) + off, dtype=torch.float64, device="cuda")
        big_c = torch.zeros(len(ci) + off, dtype=torch.int32, device="cuda")
        big_v[off:] = A.d_val
        big_c[off:] = A.d_ci
        A.close()
        import ctypes
        from monolish_b200 import _abi
        plan = ctypes.c_void_p()
        lib = handle.lib
        _abi.check(lib.mlsh_csr_plan_create(handle.h, n, n, len(v), A.d_rp.data_ptr(),
                                            big_c[off:].data_ptr(), big_v[off:].data_ptr(),
                                            _abi.F64, rp.ctypes.data_as(ctypes.c_void_p), 1,
                                            ctypes.byref(plan)), "plan")
        dx = torch.from_numpy(x).cuda()
        dy = torch.empty(n, dtype=torch.float64, device="cuda")
        _abi.check(lib.mlsh_spmv(handle.h, plan, 1.0, dx.data_ptr(), 0.0, dy.data_ptr()), "spmv")
        handle.sync()
        lib.mlsh_csr_plan_destroy(plan)
        check(rp, ci, v, x, dy.cpu().numpy(), ref)


def test_invalid_csr_rejected(handle):
    import ctypes
    import torch
    from monolish_b200 import _abi
    rp = np.array([0, 2, 1], np.int32)  # not monotone
    d = torch.zeros(4, dtype=torch.int32, device="cuda")
    dv = torch.zeros(4, dtype=torch.float64, device="cuda")
    plan = ctypes.c_void_p()
    st = handle.lib.mlsh_csr_plan_create(handle.h, 2, 2, 1, d.data_ptr(), d.data_ptr(),
                                         dv.data_ptr(), _abi.F64,
                                         rp.ctypes.data_as(ctypes.c_void_p), 1,
                                         ctypes.byref(plan))
    assert st == _abi.ERR_INVALID_CSR
    # column out of range, found by validation
    rp = np.array([0, 1, 2], np.int32)
    drp = torch.from_numpy(rp).cuda()
    dci = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
    st = handle.lib.mlsh_csr_plan_create(handle.h, 2, 2, 2, drp.data_ptr(), dci.data_ptr(),
                                         dv.data_ptr(), _abi.F64,
                                         rp.ctypes.data_as(ctypes.c_void_p), 1,
                                         ctypes.byref(plan))
    assert st == _abi.ERR_INVALID_CSR


def test_every_variant_and_autotune(handle, restatement):
    """All SpMV kernel variants give the oracle's bits on short rows and
    agree bitwise with each other; the autotuner keeps a valid variant."""
    import torch
    from monolish_b200.device import Crs
    cases = [W.poisson3d(24), W.zipf(30000, seed=5, maxlen=9000)]
    for n, rp, ci, v in cases:
        x = W.uniform_mt(n, -1, 1, 3)
        ref = restatement.spmv(rp, ci, v, x)
        A = Crs(handle, n, n, rp, ci, v)
        dx = torch.from_numpy(x).cuda()
        outs = []
        _, nvar = A.variant()
        assert nvar >= 2
        for var in range(nvar):
            A.set_variant(var)
            dy = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
            A.matvec(dx, dy)
            handle.sync()
            outs.append(dy.cpu().numpy())
            check(rp, ci, v, x, outs[-1], ref)
        for o in outs[1:]:
            assert np.array_equal(o, outs[0])
        dy = torch.empty(n, dtype=torch.float64, device="cuda")
        chosen, sec = A.autotune(dx, dy)
        assert 0 <= chosen < nvar and sec > 0
        assert A.variant()[0] == chosen
        A.close()


def test_repeatable_bitwise(handle):
    n, rp, ci, v = W.zipf(50000, seed=2, maxlen=10000)
    x = W.uniform_mt(n, -1, 1, 6)
    y1 = run_spmv(handle, n, n, rp, ci, v, x)
    y2 = run_spmv(handle, n, n, rp, ci, v, x)
    assert np.array_equal(y1, y2)


def test_diag(handle):
    import torch
    from monolish_b200.device import Crs
    n, rp, ci, v = W.convdiff3d(12, peclet=5.0)
    A = Crs(handle, n, n, rp, ci, v)
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    A.diag(d)
    handle.sync()
    ref = np.array([v[rp[i]:rp[i + 1]][ci[rp[i]:rp[i + 1]] == i][0] for i in range(n)])
    assert np.array_equal(d.cpu().numpy(), ref)


def test_short_row_limits_and_autotune(handle, restatement):
    """Every short-row limit (8, 16, 32) sums rows up to the limit in the
    reference's order (bit-identical) and the rest within the summation
    bound; the autotuner picks a (variant, limit) pair from the timings and
    keeps it; on a stencil matrix (rows of <= 7 entries) only the limit 8 is
    timed."""
    import torch
    from monolish_b200.device import Crs
    n, rp, ci, v = W.zipf(60000, seed=5, maxlen=3000)
    x = W.uniform_mt(n, -1, 1, 3)
    y_ref = restatement.spmv(rp, ci, v, x)
    lens = np.diff(rp)
    A = Crs(handle, n, n, rp, ci, v)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    for lim in (8, 16, 32):
        A.set_short_rows(lim)
        dy.fill_(float("nan"))
        A.matvec(dx, dy)
        handle.sync()
        y = dy.cpu().numpy()
        assert np.array_equal(y[lens <= lim], y_ref[lens <= lim]), lim
        check(rp, ci, v, x, y, y_ref)
    variant, _ = A.autotune(dx, dy)
    v_used, lim = A.tuning()
    assert v_used == variant and lim in (8, 16, 32)
    A.close()
    n, rp, ci, v = W.poisson3d(24)
    A = Crs(handle, n, n, rp, ci, v)
    dx = torch.from_numpy(W.uniform_mt(n, -1, 1, 4)).cuda()
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    A.autotune(dx, dy)
    assert A.tuning()[1] == 8
    A.close()
