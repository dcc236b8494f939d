"""Plain CG / BiCGSTAB on the GPU against the reference (golden fixtures)
and the oracle.

Bars: status codes equal; iteration counts within +-2% (BiCGSTAB on a
symmetric matrix: +-10%, see tests/test_oracle.py); the true relative
residual ||b - A x|| / ||b||, recomputed in FP64 on the host, below the
requested 1e-10; x within 1e-8 (relative, 2-norm) of the reference's x.
"""
import os

import numpy as np
import pytest

from monolish_b200 import workloads as W
from monolish_b200 import _abi

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def solve(handle, solver, rp, ci, v, b, x0, tol, maxiter, **kw):
    import torch
    from monolish_b200 import device as D
    n = len(rp) - 1
    A = D.Crs(handle, n, n, rp, ci, v)
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    dx = torch.from_numpy(np.ascontiguousarray(x0)).cuda()
    fn = D.cg_solve if solver == "cg" else D.bicgstab_solve
    r = fn(A, db, dx, tol, maxiter, **kw)
    x = dx.cpu().numpy()
    A.close()
    return r, x


ENGINES = {"kernels-graph": dict(engine=_abi.ENGINE_KERNELS, use_graph=True),
           "kernels-eager": dict(engine=_abi.ENGINE_KERNELS, use_graph=False),
           "cluster": dict(engine=_abi.ENGINE_CLUSTER)}


@pytest.mark.parametrize("name,solver", [("poisson16", "cg"), ("poisson16", "bicgstab"),
                                         ("poisson128", "cg"), ("convdiff10", "bicgstab")])
@pytest.mark.parametrize("engine", sorted(ENGINES))
def test_golden_solves(handle, restatement, name, solver, engine):
    g = golden(name)
    rp, ci, v, b = g["rp"], g["ci"], g["v"], g["b"]
    tol = float(g["tol"])
    r, x = solve(handle, solver, rp, ci, v, b, np.zeros_like(b), tol, 2000, **ENGINES[engine])
    gst, git, gres = g[solver]
    assert r.status == int(gst) == 0
    slack = 0.10 if (solver == "bicgstab" and name.startswith("poisson")) else 0.02
    assert abs(r.iters - int(git)) <= max(1, int(slack * git)), (r.iters, int(git))
    assert restatement.true_relres(rp, ci, v, b, x) < 1e-10
    gx = g[f"{solver}_x"]
    assert np.linalg.norm(x - gx) <= 1e-8 * np.linalg.norm(gx)
    assert r.resid < tol


@pytest.mark.parametrize("engine", sorted(ENGINES))
def test_poisson128_cg_matches_reference_exactly(handle, engine):
    """The 128x128 Jacobi-CG workload: 382 iterations, as the reference."""
    g = golden("poisson128")
    r, x = solve(handle, "cg", g["rp"], g["ci"], g["v"], g["b"], np.zeros(16384),
                 float(g["tol"]), 2000, **ENGINES[engine])
    assert r.status == 0 and r.iters == 382


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
@pytest.mark.parametrize("rows", [1024, 2048, 4096])
def test_cluster_partitions(handle, restatement, solver, rows):
    """The cluster engine on 16, 8 and 4 CTAs (rows per CTA 1024..4096)."""
    if solver == "cg":
        g = golden("poisson128")
        rp, ci, v, b = g["rp"], g["ci"], g["v"], g["b"]
        tol = float(g["tol"])
        want = int(g["cg"][1])
    else:
        n, rp, ci, v = W.convdiff3d(24, peclet=10.0)
        b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1, 1, 2))
        tol = 1e-10 * np.linalg.norm(b)
        want = restatement.bicgstab(rp, ci, v, b, np.zeros(n), tol, 3000)[1]
    r, x = solve(handle, solver, rp, ci, v, b, np.zeros_like(b), tol, 3000,
                 engine=_abi.ENGINE_CLUSTER, cluster_rows=rows)
    assert r.status == 0
    assert abs(r.iters - want) <= max(1, int(0.02 * want))
    assert restatement.true_relres(rp, ci, v, b, x) < 1e-10


def test_cluster_rejects_too_large(handle):
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v = W.poisson2d(400)  # 160,000 rows > 16 CTAs x 8192
    A = D.Crs(handle, n, n, rp, ci, v)
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(_abi.MlshError):
        D.cg_solve(A, d, d, 1e-8, 10, engine=_abi.ENGINE_CLUSTER)
    A.close()


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
def test_history_both_engines(handle, restatement, solver):
    n, rp, ci, v = W.vardiff2d(40, 33, 3, 2)
    b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1, 1, 4))
    tol = 1e-10 * np.linalg.norm(b)
    out = {}
    for name in ("kernels-graph", "cluster"):
        hist = np.full(5000, np.nan)
        r, _ = solve(handle, solver, rp, ci, v, b, np.zeros(n), tol, 5000, history=hist,
                     **ENGINES[name])
        assert r.status == 0
        h = hist[:r.iters]
        assert np.isfinite(h).all() and np.isnan(hist[r.iters:]).all()
        assert h[-1] == r.resid and h[-1] < tol
        out[name] = (r.iters, h)
    (i1, h1), (i2, h2) = out["kernels-graph"], out["cluster"]
    assert abs(i1 - i2) <= max(1, int(0.02 * i1))
    # the engines sum in different orders; the early history agrees closely
    k = min(i1, i2, 15)
    np.testing.assert_allclose(h1[:k], h2[:k], rtol=1e-6)


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
@pytest.mark.parametrize("pre", [0, 1])
@pytest.mark.parametrize("prec", ["d", "s"])
def test_reference_test_matrix(handle, solver, pre, prec):
    """The reference's own solver test (test/equation/iterative/equation_kernel.hpp)."""
    g = golden("tridiag3")
    dt = np.float64 if prec == "d" else np.float32
    tol = 1e-8 if prec == "d" else 1e-4
    r, x = solve(handle, solver, g["rp"], g["ci"], g["v"].astype(dt), g["b"].astype(dt),
                 g["x0"].astype(dt), tol, 10000, precond=pre)
    gst, git, _ = g[f"{solver}_p{pre}_{prec}"]
    assert r.status == int(gst) and r.iters == int(git)
    np.testing.assert_allclose(x, np.ones(3), rtol=10 * tol)


def test_bicgstab_convdiff_vs_oracle(handle, restatement):
    n, rp, ci, v = W.convdiff3d(24, peclet=10.0)
    b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1, 1, 2))
    tol = 1e-10 * np.linalg.norm(b)
    st, it, res, xo = restatement.bicgstab(rp, ci, v, b, np.zeros(n), tol, 3000)
    r, x = solve(handle, "bicgstab", rp, ci, v, b, np.zeros(n), tol, 3000)
    assert r.status == st == 0
    assert abs(r.iters - it) <= max(1, int(0.02 * it))
    assert restatement.true_relres(rp, ci, v, b, x) < 1e-10


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
@pytest.mark.parametrize("engine", ["kernels-graph", "cluster"])
def test_status_codes_match_oracle(handle, restatement, solver, engine):
    kw = ENGINES[engine]
    n, rp, ci, v = W.poisson2d(8)
    # b = 0, x0 = 0: CG -> NaN residual, BiCGSTAB -> breakdown
    st, it, _, _ = getattr(restatement, solver)(rp, ci, v, np.zeros(n), np.zeros(n), 1e-10, 100)
    r, _ = solve(handle, solver, rp, ci, v, np.zeros(n), np.zeros(n), 1e-10, 100, **kw)
    assert (r.status, r.iters) == (st, it)
    # maxiter
    b = restatement.spmv(rp, ci, v, np.ones(n))
    r, _ = solve(handle, solver, rp, ci, v, b, np.zeros(n), 1e-30, 5, **kw)
    assert (r.status, r.iters) == (_abi.SOLVER_MAXITER, 5)
    # NaN in b
    bn = b.copy()
    bn[3] = np.nan
    st, it, _, _ = getattr(restatement, solver)(rp, ci, v, bn, np.zeros(n), 1e-10, 100)
    r, _ = solve(handle, solver, rp, ci, v, bn, np.zeros(n), 1e-10, 100, **kw)
    assert (r.status, r.iters) == (st, it)
    # miniter holds the loop open past convergence
    n, rp, ci, v = W.poisson2d(30)
    b = restatement.spmv(rp, ci, v, np.ones(n))
    t = 0.5 * np.linalg.norm(b)
    st, it, _, _ = getattr(restatement, solver)(rp, ci, v, b, np.zeros(n), t, 100, miniter=25)
    r, _ = solve(handle, solver, rp, ci, v, b, np.zeros(n), t, 100, miniter=25, **kw)
    assert (r.status, r.iters) == (st, it) == (0, 25)
    # maxiter = 0
    r, _ = solve(handle, solver, rp, ci, v, b, np.zeros(n), 1e-3, 0, **kw)
    assert r.status == _abi.SOLVER_MAXITER and r.iters == 0


def test_zero_diagonal_jacobi_gives_nan_status(handle, restatement):
    """Host-side fault injection: a zero on the diagonal makes Jacobi 1/0."""
    n, rp, ci, v = W.poisson2d(8)
    v = v.copy()
    dmask = ci == np.repeat(np.arange(n), np.diff(rp))
    idx = np.nonzero(dmask)[0][5]
    v[idx] = 0.0
    b = np.ones(n)
    st, it, _, _ = restatement.cg(rp, ci, v, b, np.zeros(n), 1e-10, 100)
    for kw in (ENGINES["kernels-graph"], ENGINES["cluster"]):
        r, _ = solve(handle, "cg", rp, ci, v, b, np.zeros(n), 1e-10, 100, **kw)
        assert (r.status, r.iters) == (st, it) == (_abi.SOLVER_RESIDUAL_NAN, 1)


def test_graph_and_eager_identical(handle):
    n, rp, ci, v = W.vardiff2d(90, 77, 3, 5)
    b = np.random.default_rng(0).uniform(-1, 1, n)
    tol = 1e-10 * np.linalg.norm(b)
    for solver in ("cg", "bicgstab"):
        kw = dict(engine=_abi.ENGINE_KERNELS)
        r1, x1 = solve(handle, solver, rp, ci, v, b, np.zeros(n), tol, 5000, use_graph=True, **kw)
        r2, x2 = solve(handle, solver, rp, ci, v, b, np.zeros(n), tol, 5000, use_graph=False,
                       **kw)
        r3, x3 = solve(handle, solver, rp, ci, v, b, np.zeros(n), tol, 5000, use_graph=True, **kw)
        assert r1.iters == r2.iters == r3.iters
        assert np.array_equal(x1, x2) and np.array_equal(x1, x3)


def test_non_square_is_size_error(handle):
    import torch
    from monolish_b200 import device as D
    rp = np.array([0, 1, 2], np.int32)
    A = D.Crs(handle, 2, 3, rp, np.array([0, 2], np.int32), np.array([1.0, 2.0]))
    d = torch.zeros(3, dtype=torch.float64, device="cuda")
    r = D.cg_solve(A, d, d, 1e-8, 10)
    assert r.status == _abi.SOLVER_SIZE_ERROR
    A.close()
