"""Device-side waits that run out: a solve whose wall-clock budget (cluster
engine, batches) or whose sweep poll bound (SOR / IC / ILU) is set tiny on
an ordinary system returns MLSH_ERR_TIMEOUT -- the kernel notices, stops on
its own and reports -- and the same handle then solves the same system
correctly.  Nothing here faults or hangs: every wait is bounded, the limits
just make the bound small.  (The reference has no counterpart: it exit()s
on a CUDA error, src/internal/monolish_internal.hpp:34-43.)"""
import numpy as np
import pytest

from monolish_b200 import _abi
from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_cluster_budget_times_out_then_solves(handle, restatement):
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v = W.poisson2d(128)
    b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1, 1, 0))
    tol = 1e-10 * np.linalg.norm(b)
    A = D.Crs(handle, n, n, rp, ci, v)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(_abi.MlshError) as ei:
        D.cg_solve(A, db, dx, tol, 2000, engine=_abi.ENGINE_CLUSTER, time_limit=1e-7)
    assert ei.value.status == _abi.ERR_TIMEOUT
    dx.zero_()
    r = D.cg_solve(A, db, dx, tol, 2000, engine=_abi.ENGINE_CLUSTER)
    assert (r.status, r.iters) == (0, 382)
    assert restatement.true_relres(rp, ci, v, b, dx.cpu().numpy()) < 1e-10
    A.close()


def test_batch_budget_times_out_then_solves(handle, restatement):
    import torch
    from monolish_b200 import device as D
    systems = []
    for k, (nx, ny) in enumerate([(40, 30), (90, 77), (120, 101)]):
        _, rp, ci, v = W.vardiff2d(nx, ny, 3, k)
        systems.append((rp, ci, v))
    bs = [restatement.spmv(rp, ci, v, W.uniform_mt(len(rp) - 1, -1, 1, 3 + k))
          for k, (rp, ci, v) in enumerate(systems)]
    tol = np.array([1e-8 * np.linalg.norm(b) for b in bs])
    B = D.Batch(handle, systems)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.zeros_like(db)
    with pytest.raises(_abi.MlshError) as ei:  # the batch's first non-success status
        B.solve("cg", db, dx, tol, 20000, time_limit=1e-7)
    assert ei.value.status == _abi.ERR_TIMEOUT
    dx.zero_()
    status, iters, _ = B.solve("cg", db, dx, tol, 20000)
    assert (status == 0).all()
    xs = np.split(dx.cpu().numpy(), np.cumsum([len(b) for b in bs])[:-1])
    for k, (rp, ci, v) in enumerate(systems):
        st, it, _, _ = restatement.cg(rp, ci, v, bs[k], np.zeros(len(bs[k])), tol[k], 20000)
        assert st == 0 and abs(iters[k] - it) <= max(1, it // 50)
        assert restatement.true_relres(rp, ci, v, bs[k], xs[k]) < 1e-8
    B.close()


@pytest.mark.parametrize("kind", ["ic", "sor"])
def test_sweep_poll_bound_times_out_then_solves(handle, restatement, kind):
    """A 3D system large enough for the multi-CTA sweeps (blocks wait on
    other blocks' flags): with one poll per wait, blocks give up and the
    solve reports MLSH_ERR_TIMEOUT; with the default bound it converges in
    the oracle's iteration count."""
    import torch
    from monolish_b200 import device as D
    n, rp, ci, v = W.poisson3d(48)
    b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1, 1, 1))
    tol = 1e-10 * np.linalg.norm(b)
    A = D.Crs(handle, n, n, rp, ci, v)
    pc = D.Precond(A, {"ic": _abi.PRECOND_IC, "sor": _abi.PRECOND_SOR}[kind])
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(_abi.MlshError) as ei:
        D.cg_solve_precond(A, pc, db, dx, tol, 30, wait_polls=1)
    assert ei.value.status == _abi.ERR_TIMEOUT
    dx.zero_()
    r = D.cg_solve_precond(A, pc, db, dx, tol, 2000)
    st, it, _, _ = restatement.cg(rp, ci, v, b, np.zeros(n), tol, 2000,
                                  precond={"ic": 3, "sor": 2}[kind])
    assert r.status == st == 0
    assert abs(r.iters - it) <= max(1, it // 50), (r.iters, it)
    assert restatement.true_relres(rp, ci, v, b, dx.cpu().numpy()) < 1e-10
    pc.close()
    A.close()
