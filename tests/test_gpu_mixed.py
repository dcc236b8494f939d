"""Mixed precision: FP32 inner iterations inside FP64 iterative refinement.

Bars (the outer loop recomputes the true residual in FP64): status SUCCESS,
true relative residual ||b - A x|| / ||b|| < 1e-10 recomputed on the host,
x within 1e-5 (relative) of the oracle's FP64 solution -- two different
iterations stopped at a 1e-10 residual differ by up to cond(A) * 1e-10 --
and an inner iteration count within 2x of the plain FP64 solve's."""
import numpy as np
import pytest

from monolish_b200 import _abi
from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu


def solve_both(handle, restatement, kind, n, rp, ci, v, seed, engine=_abi.ENGINE_AUTO):
    import torch
    from monolish_b200 import device as D
    xt = W.uniform_mt(n, -1, 1, seed)
    b = restatement.spmv(rp, ci, v, xt)
    tol = 1e-10 * np.linalg.norm(b)
    A = D.Crs(handle, n, n, rp, ci, v)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    mixed = D.cg_solve_mixed if kind == "cg" else D.bicgstab_solve_mixed
    plain = D.cg_solve if kind == "cg" else D.bicgstab_solve
    hist = np.full(100, np.nan)
    rm = mixed(A, db, dx, tol, 20000, inner_tol=1e-4, history=hist, engine=engine)
    xm = dx.cpu().numpy()
    dx.zero_()
    rpl = plain(A, db, dx, tol, 20000)
    A.close()
    st, it, _, xo = getattr(restatement, kind)(rp, ci, v, b, np.zeros(n), tol, 20000)
    return rm, xm, rpl, st, it, xo, b, hist


@pytest.mark.parametrize("engine", [_abi.ENGINE_AUTO, _abi.ENGINE_KERNELS],
                         ids=["auto", "kernels"])
@pytest.mark.parametrize("case", ["convdiff40", "convdiff64_pe2"])
def test_mixed_bicgstab_convdiff(handle, restatement, case, engine):
    """AUTO runs these sizes' FP32 iterations on the cluster engine
    (restarted refinement); KERNELS on the kernel engine (reliable
    updates, the path large systems take)."""
    m, pe = (40, 10.0) if case == "convdiff40" else (64, 2.0)
    n, rp, ci, v = W.convdiff3d(m, peclet=pe)
    rm, xm, rpl, st, it, xo, b, hist = solve_both(handle, restatement, "bicgstab", n, rp, ci,
                                                  v, 2, engine)
    assert rm.status == 0 and st == 0 and rpl.status == 0
    assert rm.outer >= 2
    assert restatement.true_relres(rp, ci, v, b, xm) < 1e-10
    assert np.linalg.norm(xm - xo) <= 1e-5 * np.linalg.norm(xo)
    assert rm.iters <= 2 * it
    # the outer history is the true residual per refinement step, decreasing
    h = hist[:rm.outer + 1]
    assert np.isfinite(h).all() and (np.diff(h) < 0).all()


def test_mixed_cg_poisson(handle, restatement):
    n, rp, ci, v = W.poisson2d(200)
    rm, xm, rpl, st, it, xo, b, _ = solve_both(handle, restatement, "cg", n, rp, ci, v, 0)
    assert rm.status == 0 and st == 0
    assert restatement.true_relres(rp, ci, v, b, xm) < 1e-10
    assert np.linalg.norm(xm - xo) <= 1e-5 * np.linalg.norm(xo)
    assert rm.iters <= 2 * it


def test_mixed_with_32bit_columns(handle, restatement):
    """A symmetrically permuted Poisson matrix: its tiles' columns span more
    than 65,536, so the FP32 plan keeps 32-bit columns."""
    n0, rp0, ci0, v0 = W.poisson2d(300)
    perm = np.random.default_rng(3).permutation(n0)
    inv = np.empty(n0, np.int64)
    inv[perm] = np.arange(n0)
    rows = []
    for new_r in range(n0):
        r = perm[new_r]
        cols = inv[ci0[rp0[r]:rp0[r + 1]]]
        order = np.argsort(cols)
        rows.append((cols[order], v0[rp0[r]:rp0[r + 1]][order]))
    rp = np.concatenate([[0], np.cumsum([len(c) for c, _ in rows])]).astype(np.int32)
    ci = np.concatenate([c for c, _ in rows]).astype(np.int32)
    v = np.concatenate([x for _, x in rows])
    rm, xm, rpl, st, it, xo, b, _ = solve_both(handle, restatement, "cg", n0, rp, ci, v, 1)
    assert rm.status == 0 and st == 0
    assert restatement.true_relres(rp, ci, v, b, xm) < 1e-10
    assert rm.iters <= 2 * it


def test_mixed_rejects_fp32_plan(handle):
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v = W.poisson2d(10)
    A = D.Crs(handle, n, n, rp, ci, v.astype(np.float32))
    d = torch.zeros(n, dtype=torch.float32, device="cuda")
    with pytest.raises(_abi.MlshError):
        D.cg_solve_mixed(A, d, d, 1e-8, 10)
    A.close()


def test_mixed_bicgstab_reliable_updates_eager_equals_graph(handle, restatement):
    """The reliable-update engine gives the same result launched as one graph
    or iteration by iteration, and takes about as many FP32 iterations as the
    plain FP64 solve takes FP64 ones."""
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v = W.convdiff3d(48, peclet=5.0)
    xt = W.uniform_mt(n, -1, 1, 4)
    b = restatement.spmv(rp, ci, v, xt)
    tol = 1e-10 * np.linalg.norm(b)
    A = D.Crs(handle, n, n, rp, ci, v)
    db = torch.from_numpy(b).cuda()
    xs, rs = [], []
    for use_graph in (True, False):
        dx = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = D.bicgstab_solve_mixed(A, db, dx, tol, 20000, inner_tol=1e-4,
                                   engine=_abi.ENGINE_KERNELS, use_graph=use_graph)
        xs.append(dx.cpu().numpy())
        rs.append(r)
    A.close()
    assert rs[0].status == 0 and (rs[0].iters, rs[0].outer) == (rs[1].iters, rs[1].outer)
    assert np.array_equal(xs[0], xs[1])
    st, it, _, _ = restatement.bicgstab(rp, ci, v, b, np.zeros(n), tol, 20000)
    assert rs[0].iters <= 1.25 * it + 10
    assert restatement.true_relres(rp, ci, v, b, xs[0]) < 1e-10


def test_mixed_bicgstab_reliable_updates_maxiter(handle, restatement):
    """Stopped by maxiter: the correction so far is applied and the status is
    MAXITER with the true residual."""
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v = W.convdiff3d(40, peclet=10.0)
    xt = W.uniform_mt(n, -1, 1, 5)
    b = restatement.spmv(rp, ci, v, xt)
    A = D.Crs(handle, n, n, rp, ci, v)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = D.bicgstab_solve_mixed(A, db, dx, 1e-10 * np.linalg.norm(b), 7, inner_tol=1e-4,
                               engine=_abi.ENGINE_KERNELS)
    A.close()
    assert r.status == _abi.SOLVER_MAXITER and r.iters == 7
    rel = restatement.true_relres(rp, ci, v, b, dx.cpu().numpy())
    assert rel < 1.0 and abs(r.resid / np.linalg.norm(b) - rel) <= 1e-6 * rel
