"""Parity at the measured sizes: the configurations the benchmark times,
run in full through the C ABI and checked against the oracle and against
summaries of the reference's own CPU build (tests/golden/fullsize.npz, made
by tests/golden/make_golden.py from oracle/_ref).

* SpMV, 3D 7-point Laplacian 256^3 (n = 16,777,216, nnz = 117,047,296) in
  FP64 and FP32: every row has <= 8 entries, so every row of y must be
  bit-identical to the reference loop (crs_matvec.hpp:101-108), checked on
  all rows against the restatement, whose output is pinned to the
  reference's at 4,096 sampled rows and by its sums.
* SpMV, Zipf(2) matrix with n = 4,194,304 (rows up to 10,000 entries), FP64
  and FP32: rows of <= 8 entries bit-identical, longer rows within
  4 * len * eps * (|A||x|)_i of the restatement (the summation error bound
  for a different association order), the restatement pinned as above.
* Jacobi-BiCGSTAB on the 160^3 convection-diffusion system (n = 4,096,000),
  plain FP64: status SUCCESS, iterations within +-2% of the reference's
  (bicgstab.cpp:53-130; 276 in the reference build), true relative residual
  recomputed in FP64 on the host below 1e-10.  Mixed FP32/FP64 at inner
  tolerance 1e-4: SUCCESS, true relative residual below 1e-10 and x within
  1e-5 (relative) of the plain FP64 solution.
* The 2,048-system diffusion batch, Jacobi-CG to 1e-8 in one persistent
  launch: every system's status equal to the reference's, its iterations
  within +-2% of the reference's (cg.cpp:46-80), its true relative residual
  below 1e-8; the mixed batch: every system SUCCESS below the true 1e-8.
"""
import os

import numpy as np
import pytest

from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def fullsize():
    return np.load(os.path.join(GOLDEN, "fullsize.npz"))


def gpu_spmv(handle, n, rp, ci, v, x):
    import torch
    from monolish_b200.device import Crs
    A = Crs(handle, n, n, rp, ci, v)
    dx = torch.from_numpy(x).cuda()
    dy = torch.full((n,), float("nan"), dtype=dx.dtype, device="cuda")
    A.matvec(dx, dy)
    handle.sync()
    y = dy.cpu().numpy()
    A.close()
    del dx, dy
    torch.cuda.empty_cache()
    return y


def pin_to_reference(g, tag, y_ref):
    rows = g[f"{tag}_rows"]
    assert np.array_equal(y_ref[rows].astype(np.float64), g[f"{tag}_y"])
    y64 = y_ref.astype(np.float64)
    assert np.array_equal(np.array([y64.sum(), np.abs(y64).sum()]), g[f"{tag}_sum"])


def check_rows(rp, ci, v, x, y, y_ref):
    lens = np.diff(rp)
    short = lens <= 8
    assert np.array_equal(y[short], y_ref[short]), "rows of <= 8 entries must match bitwise"
    if (~short).any():
        row_of = np.repeat(np.arange(len(lens)), lens)
        absax = np.bincount(row_of, weights=np.abs(v.astype(np.float64) * x[ci]),
                            minlength=len(lens))
        bound = 4 * lens * np.finfo(v.dtype).eps * absax
        err = np.abs(y.astype(np.float64) - y_ref.astype(np.float64))
        bad = np.nonzero(~short & (err > bound))[0]
        assert bad.size == 0, (bad[:5], err[bad[:5]], bound[bad[:5]])


@pytest.mark.parametrize("sfx", ["d", "s"])
def test_spmv_laplacian256_bitwise(handle, restatement, fullsize, sfx):
    dt = np.float64 if sfx == "d" else np.float32
    n, rp, ci, v = W.poisson3d(256)
    v = v.astype(dt)
    x = W.uniform_fast(n, -1.0, 1.0, 1).astype(dt)
    y_ref = restatement.spmv(rp, ci, v, x)
    pin_to_reference(fullsize, f"lap256_{sfx}", y_ref)
    y = gpu_spmv(handle, n, rp, ci, v, x)
    assert np.array_equal(y, y_ref)


@pytest.mark.parametrize("sfx", ["d", "s"])
def test_spmv_zipf4m(handle, restatement, fullsize, sfx):
    dt = np.float64 if sfx == "d" else np.float32
    n, rp, ci, v = W.zipf(4194304, seed=1)
    assert np.diff(rp).max() > 1792  # rows split across tiles are part of the case
    v = v.astype(dt)
    x = W.uniform_fast(n, -1.0, 1.0, 1).astype(dt)
    y_ref = restatement.spmv(rp, ci, v, x)
    pin_to_reference(fullsize, f"zipf4m_{sfx}", y_ref)
    y = gpu_spmv(handle, n, rp, ci, v, x)
    check_rows(rp, ci, v, x, y, y_ref)


@pytest.fixture(scope="module")
def convdiff160(restatement, fullsize):
    n, rp, ci, v = W.convdiff3d(160, peclet=10.0)
    b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1.0, 1.0, 2))
    assert np.array_equal(np.array([b.sum(), np.abs(b).sum()]), fullsize["convdiff160_b_sum"])
    return n, rp, ci, v, b


def test_bicgstab_convdiff160_plain_and_mixed(handle, restatement, fullsize, convdiff160):
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v, b = convdiff160
    st_ref, it_ref, _, relres_ref, nb = fullsize["convdiff160_bicgstab"]
    tol = 1e-10 * float(np.linalg.norm(b))
    assert tol == pytest.approx(1e-10 * nb, rel=1e-14)
    A = D.Crs(handle, n, n, rp, ci, v)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = D.bicgstab_solve(A, db, dx, tol, 20000)
    x_plain = dx.cpu().numpy()
    assert r.status == int(st_ref) == 0
    assert abs(r.iters - int(it_ref)) <= max(1, int(0.02 * it_ref)), (r.iters, int(it_ref))
    assert restatement.true_relres(rp, ci, v, b, x_plain) < 1e-10
    dx.zero_()
    rm = D.bicgstab_solve_mixed(A, db, dx, tol, 20000, inner_tol=1e-4)
    x_mixed = dx.cpu().numpy()
    A.close()
    assert rm.status == 0 and rm.outer >= 2
    assert restatement.true_relres(rp, ci, v, b, x_mixed) < 1e-10
    assert np.linalg.norm(x_mixed - x_plain) <= 1e-5 * np.linalg.norm(x_plain)


@pytest.fixture(scope="module")
def batch2048(restatement):
    systems = W.diffusion_batch(2048, seed=3)
    bs = [restatement.spmv(rp, ci, v, W.uniform_mt(len(rp) - 1, -1.0, 1.0, 3 + k))
          for k, (rp, ci, v) in enumerate(systems)]
    return systems, bs


def _run_batch(handle, systems, bs, tol, mixed):
    import torch
    from monolish_b200 import device as D
    B = D.Batch(handle, systems)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.zeros_like(db)
    if mixed:
        status, iters, resid = B.solve_mixed(db, dx, tol, 20000, inner_tol=1e-2)
    else:
        status, iters, resid = B.solve("cg", db, dx, tol, 20000)
    xs = np.split(dx.cpu().numpy(), np.cumsum([len(b) for b in bs])[:-1])
    B.close()
    return status, iters, resid, xs


def test_batch2048_cg_matches_reference(handle, restatement, fullsize, batch2048):
    systems, bs = batch2048
    g = fullsize["batch2048_cg"]
    nb = np.array([np.linalg.norm(b) for b in bs])
    np.testing.assert_allclose(nb, g[:, 3], rtol=1e-14)
    tol = 1e-8 * nb
    status, iters, resid, xs = _run_batch(handle, systems, bs, tol, mixed=False)
    assert np.array_equal(status, g[:, 0].astype(np.int32))
    it_ref = g[:, 1].astype(np.int64)
    off = np.abs(iters - it_ref) > np.maximum(1, (0.02 * it_ref).astype(np.int64))
    assert not off.any(), (np.nonzero(off)[0][:5], iters[off][:5], it_ref[off][:5])
    rel = np.array([restatement.true_relres(rp, ci, v, bs[k], xs[k])
                    for k, (rp, ci, v) in enumerate(systems)])
    assert (rel < 1e-8).all(), (rel.argmax(), rel.max())


def test_batch2048_mixed_reaches_true_tolerance(handle, restatement, batch2048):
    systems, bs = batch2048
    tol = 1e-8 * np.array([np.linalg.norm(b) for b in bs])
    status, iters, resid, xs = _run_batch(handle, systems, bs, tol, mixed=True)
    assert (status == 0).all(), np.nonzero(status)[0][:5]
    rel = np.array([restatement.true_relres(rp, ci, v, bs[k], xs[k])
                    for k, (rp, ci, v) in enumerate(systems)])
    # the FP64 refresh stops at the true residual; host recomputation differs
    # from the device's by rounding only
    assert (rel < 1e-8 * (1 + 1e-6)).all(), (rel.argmax(), rel.max())
