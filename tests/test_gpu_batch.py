"""Batched solves (one persistent launch per cluster-size group) against the
oracle, system by system: every status equal, iteration counts within
+-2% (BiCGSTAB: +-10% on these symmetric-part-dominated small systems),
true relative residual below the requested tolerance x 10, and the same
result for a system whether it is solved alone or in the batch."""
import numpy as np
import pytest

from monolish_b200 import _abi
from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu


def make_systems(sizes, seed):
    systems = []
    for k, n in enumerate(sizes):
        nx, ny = W.grid2d_for(int(n))
        _, rp, ci, v = W.vardiff2d(nx, ny, seed, k)
        systems.append((rp, ci, v))
    return systems


def run_batch(handle, systems, kind, rel_tol, maxiter, restatement, x_seed=5):
    import torch
    from monolish_b200 import device as D
    B = D.Batch(handle, systems)
    bs, xts = [], []
    for k, (rp, ci, v) in enumerate(systems):
        xt = W.uniform_mt(len(rp) - 1, -1, 1, x_seed + k)
        xts.append(xt)
        bs.append(restatement.spmv(rp, ci, v, xt))
    b_all = np.concatenate(bs)
    tol = np.array([rel_tol * np.linalg.norm(b) for b in bs])
    db = torch.from_numpy(b_all).cuda()
    dx = torch.zeros_like(db)
    status, iters, resid = B.solve(kind, db, dx, tol, maxiter)
    x_all = dx.cpu().numpy()
    B.close()
    xs = np.split(x_all, np.cumsum([len(b) for b in bs])[:-1])
    return status, iters, resid, xs, bs, tol


def convdiff_systems(count, seed):
    """Nonsymmetric systems for BiCGSTAB: upwind convection-diffusion on
    m^3 grids (m in 2..24) with cell Peclet numbers in [0, 20]."""
    rng = np.random.default_rng(seed)
    systems = []
    for _ in range(count):
        m = int(rng.integers(2, 25))
        _, rp, ci, v = W.convdiff3d(m, peclet=float(rng.uniform(0, 20)))
        systems.append((rp, ci, v))
    return systems


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_batch_matches_oracle(handle, restatement, kind):
    if kind == "cg":
        rng = np.random.default_rng(7)
        sizes = np.exp(rng.uniform(np.log(40), np.log(30000), 60)).round().astype(int)
        sizes[:3] = [1, 2, 20000]  # tiny and multi-CTA systems
        systems = make_systems(sizes, seed=3)
    else:
        systems = convdiff_systems(40, seed=9)
    status, iters, resid, xs, bs, tol = run_batch(handle, systems, kind, 1e-8, 5000,
                                                   restatement)
    slack = 0.02
    for k, (rp, ci, v) in enumerate(systems):
        st, it, _, _ = getattr(restatement, kind)(rp, ci, v, bs[k], np.zeros(len(bs[k])),
                                                  tol[k], 5000)
        assert status[k] == st, (k, status[k], st)
        if st != 0:  # e.g. BiCGSTAB on a 1x1 system: exact after one step, then 0/0
            assert iters[k] == it
            continue
        assert abs(iters[k] - it) <= max(1, int(slack * it)), (k, iters[k], it)
        assert resid[k] < tol[k]
        assert restatement.true_relres(rp, ci, v, bs[k], xs[k]) < 1e-7


def test_batch_same_as_alone(handle, restatement):
    """A system's result does not depend on the batch it is in."""
    import torch
    from monolish_b200 import device as D
    sizes = [500, 3000, 9000, 17000]
    systems = make_systems(sizes, seed=11)
    status, iters, resid, xs, bs, tol = run_batch(handle, systems, "cg", 1e-8, 5000,
                                                   restatement)
    # the third system alone, as a batch of one and as a single solve
    k = 2
    s1, i1, r1, x1, _, _ = run_batch(handle, [systems[k]], "cg", 1e-8, 5000, restatement,
                                     x_seed=5 + k)
    assert (s1[0], i1[0]) == (status[k], iters[k])
    assert np.array_equal(x1[0], xs[k])
    rp, ci, v = systems[k]
    A = D.Crs(handle, len(rp) - 1, len(rp) - 1, rp, ci, v)
    dx = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    # the batch runs a 9,000-row CG system on 2 CTAs of 8,192 rows
    r = D.cg_solve(A, torch.from_numpy(bs[k]).cuda(), dx, tol[k], 5000,
                   engine=_abi.ENGINE_CLUSTER, cluster_rows=8192)
    A.close()
    assert (r.status, r.iters) == (status[k], iters[k])
    assert np.array_equal(dx.cpu().numpy(), xs[k])


def test_batch_statuses_per_system(handle, restatement):
    """Systems fail independently: a NaN right-hand side in one system and
    a too-small maxiter do not disturb the others."""
    import torch
    from monolish_b200 import device as D
    systems = make_systems([800, 1200, 2500], seed=13)
    B = D.Batch(handle, systems)
    bs = [restatement.spmv(rp, ci, v, np.ones(len(rp) - 1)) for rp, ci, v in systems]
    bs[1][7] = np.nan
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.zeros_like(db)
    status, iters, resid = B.solve("cg", db, dx, 1e-8, 3000)
    assert status[0] == 0 and status[2] == 0
    assert status[1] == _abi.SOLVER_RESIDUAL_NAN
    dx.zero_()
    status, iters, resid = B.solve("cg", db, dx, 1e-8, 3)
    assert (status[[0, 2]] == _abi.SOLVER_MAXITER).all() and (iters[[0, 2]] == 3).all()
    B.close()


def test_batch_mixed_cg(handle, restatement):
    """Mixed-precision batch (FP32 iterations, FP64 refreshes every 1e-2):
    every system reaches the requested true residual, in about as many
    iterations as the FP64 oracle, and its result does not depend on the
    batch it is in."""
    import torch
    from monolish_b200 import device as D
    rng = np.random.default_rng(17)
    sizes = np.exp(rng.uniform(np.log(40), np.log(30000), 40)).round().astype(int)
    sizes[:3] = [1, 2, 20000]
    systems = make_systems(sizes, seed=19)
    bs, tol = [], []
    for k, (rp, ci, v) in enumerate(systems):
        b = restatement.spmv(rp, ci, v, W.uniform_mt(len(rp) - 1, -1, 1, 31 + k))
        bs.append(b)
        tol.append(1e-8 * np.linalg.norm(b))
    B = D.Batch(handle, systems)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.zeros_like(db)
    status, iters, resid = B.solve_mixed(db, dx, np.array(tol), 20000, inner_tol=1e-2)
    xs = np.split(dx.cpu().numpy(), np.cumsum([len(b) for b in bs])[:-1])
    for k, (rp, ci, v) in enumerate(systems):
        assert status[k] == 0, (k, status[k])
        rel = restatement.true_relres(rp, ci, v, bs[k], xs[k])
        assert rel < 1e-8 * 1.0000001 and abs(resid[k] - rel * np.linalg.norm(bs[k])) <= \
            1e-6 * resid[k] + 1e-300
        st, it, _, _ = restatement.cg(rp, ci, v, bs[k], np.zeros(len(bs[k])), tol[k], 20000)
        assert iters[k] <= 1.3 * it + 5, (k, iters[k], it)
    # one system alone: same iterations and bits
    k = 2
    B1 = D.Batch(handle, [systems[k]])
    db1 = torch.from_numpy(bs[k]).cuda()
    dx1 = torch.zeros_like(db1)
    s1, i1, r1 = B1.solve_mixed(db1, dx1, tol[k], 20000, inner_tol=1e-2)
    assert (s1[0], i1[0]) == (status[k], iters[k])
    assert np.array_equal(dx1.cpu().numpy(), xs[k])
    B.close()
    B1.close()


def test_batch_autotune(handle, restatement):
    """The autotuner times one solve per rows-per-CTA cap, keeps the fastest,
    leaves the initial guess as it found it, and the batch solves to the
    oracle's statuses and iteration counts (+-2%) under the chosen cap."""
    import torch
    from monolish_b200 import device as D
    systems = make_systems([500, 3000, 9000, 17000, 30000, 60000], seed=23)
    bs, x0s = [], []
    for k, (rp, ci, v) in enumerate(systems):
        bs.append(restatement.spmv(rp, ci, v, W.uniform_mt(len(rp) - 1, -1, 1, 41 + k)))
        x0s.append(W.uniform_mt(len(rp) - 1, -0.1, 0.1, 61 + k))
    tol = np.array([1e-8 * np.linalg.norm(b) for b in bs])
    B = D.Batch(handle, systems)
    assert B.info("cg")[0] == 16384
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    x0 = torch.from_numpy(np.concatenate(x0s)).cuda()
    dx = x0.clone()
    cap, secs = B.autotune("cg", db, dx, tol, 5000)
    assert cap in (1024, 2048, 4096, 8192, 16384) and secs > 0
    assert torch.equal(dx, x0)
    assert B.info("cg")[0] == cap and B.info("cg")[1] >= 1
    status, iters, resid = B.solve("cg", db, dx, tol, 5000)
    xs = np.split(dx.cpu().numpy(), np.cumsum([len(b) for b in bs])[:-1])
    for k, (rp, ci, v) in enumerate(systems):
        st, it, _, _ = restatement.cg(rp, ci, v, bs[k], x0s[k], tol[k], 5000)
        assert status[k] == st == 0
        assert abs(iters[k] - it) <= max(1, it // 50), (k, iters[k], it)
        assert restatement.true_relres(rp, ci, v, bs[k], xs[k]) < 1e-7
    B.close()


def test_batch_repeats_bitwise(handle, restatement):
    """Every reduction of the cluster engine has a fixed order, so solving the
    same batch again gives the same bits; repeats of the 2,048-system batch
    (the size at which CTAs of one cluster drift furthest apart between
    barriers) must agree exactly in x, statuses and iteration counts."""
    import torch
    from monolish_b200 import device as D
    systems = W.diffusion_batch(2048, seed=3)
    bs = [restatement.spmv(rp, ci, v, W.uniform_mt(len(rp) - 1, -1.0, 1.0, 3 + k))
          for k, (rp, ci, v) in enumerate(systems)]
    tol = np.array([1e-8 * np.linalg.norm(b) for b in bs])
    B = D.Batch(handle, systems)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.zeros_like(db)
    first = None
    for _ in range(6):
        dx.zero_()
        status, iters, _ = B.solve("cg", db, dx, tol, 20000)
        got = (dx.cpu().numpy(), status.copy(), iters.copy())
        if first is None:
            first = got
            assert (status == 0).all()
        else:
            assert np.array_equal(got[1], first[1]) and np.array_equal(got[2], first[2])
            assert np.array_equal(got[0], first[0])
    B.close()
