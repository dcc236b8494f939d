"""SOR / IC(0) / ILU(0) on the GPU against the oracle and the reference.

Bars:
  * factorizations (IC / ILU values, SOR multipliers): bit-identical to the
    oracle's sequential restatement (same operations, same order);
  * zero pivots: the same row as the oracle;
  * apply z = M^{-1} r: blocks whose rows depend only on the adjacent row
    inside the block are resolved by an affine scan and the backward sweep
    sums a row's entries in another order, so z agrees with the sequential
    sweeps to 1e-12 (FP64) / 1e-5 (FP32) relative (max-norm); SOR apply
    against the reference build itself; systems both below and above the
    single-CTA size (solution and schedule within 200 KB of shared memory);
  * preconditioned CG / BiCGSTAB and the SOR solver: same status, iteration
    counts within +-1 (FP64) / +-10% (FP32), x within 1e-8 (FP64) relative.
"""
import numpy as np
import pytest

from monolish_b200 import _abi
from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu

SOR, IC, ILU = _abi.PRECOND_SOR, _abi.PRECOND_IC, _abi.PRECOND_ILU


def random_sparse(n, per_row, seed, symmetric=False, long_rows=0, long_len=300):
    """Diagonally dominant CRS with sorted rows; `long_rows` rows get
    `long_len` entries spread over the whole range."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = long_len if i < long_rows else per_row
        cols = rng.choice(n, size=min(k, n), replace=False)
        rows.append(set(int(c) for c in cols if c != i))
    if symmetric:
        for i in range(n):
            for c in list(rows[i]):
                rows[c].add(i)
    rp = [0]
    ci, v = [], []
    vals = {}
    for i in range(n):
        cols = sorted(rows[i] | {i})
        for c in cols:
            if c == i:
                continue
            key = (min(i, c), max(i, c)) if symmetric else (i, c)
            if key not in vals:
                vals[key] = rng.uniform(-1, 1)
        off = sum(abs(vals[(min(i, c), max(i, c)) if symmetric else (i, c)])
                  for c in cols if c != i)
        for c in cols:
            ci.append(c)
            if c == i:
                v.append(off + 1.0)
            else:
                v.append(vals[(min(i, c), max(i, c)) if symmetric else (i, c)])
        rp.append(len(ci))
    return (np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64))


def matrices():
    out = {"poisson2d_40x37": W.poisson2d(40, 37)[1:],
           "poisson3d_12": W.poisson3d(12)[1:],
           "random_1000": random_sparse(1000, 6, 1),
           "random_long": random_sparse(777, 4, 2, long_rows=5),
           "spd_random_900": random_sparse(900, 5, 3, symmetric=True),
           "tiny_5": random_sparse(5, 2, 4),
           "one": (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([4.0])),
           # solutions larger than 200 KB in both precisions: the multi-CTA
           # (flag-synchronized) sweeps instead of the single-CTA ones
           "poisson2d_240": W.poisson2d(240)[1:],
           "random_60k": random_sparse(60000, 4, 6, long_rows=3)}
    return out


MATS = matrices()
SYM = {"poisson2d_40x37", "poisson3d_12", "spd_random_900", "one", "poisson2d_240"}


def crs(handle, rp, ci, v):
    from monolish_b200 import device as D
    n = len(rp) - 1
    return D.Crs(handle, n, n, rp, ci, v)


def cu(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("kind", [SOR, IC, ILU])
@pytest.mark.parametrize("name", sorted(MATS))
def test_factor_and_apply(handle, restatement, name, kind, dtype):
    from monolish_b200 import device as D
    if kind == IC and name not in SYM:
        pytest.skip("IC needs a symmetric matrix")
    rp, ci, v = MATS[name]
    v = v.astype(dtype)
    n = len(rp) - 1
    A = crs(handle, rp, ci, v)
    pc = D.Precond(A, kind, omega=1.9)
    want_f, want_piv = restatement.precond_factor(rp, ci, v, kind, omega=1.9)
    got_f = pc.factor().cpu().numpy()
    assert np.array_equal(got_f, want_f), np.abs(got_f - want_f).max()
    assert pc.zero_pivot()[0] == want_piv
    r = np.random.default_rng(7).uniform(-1, 1, n).astype(dtype)
    dz = cu(np.zeros(n, dtype))
    pc.apply(cu(r), dz)
    got = dz.cpu().numpy()
    want = restatement.precond_apply(rp, ci, v, kind, r, omega=1.9)
    assert rel_err(got, want) < (1e-12 if dtype == np.float64 else 1e-5)
    pc.close()
    A.close()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_sor_apply_matches_reference(handle, reference, dtype):
    from monolish_b200 import device as D
    rp, ci, v = W.poisson3d(16)[1:]
    v = v.astype(dtype)
    n = len(rp) - 1
    A = crs(handle, rp, ci, v)
    pc = D.Precond(A, SOR, omega=1.9)
    r = np.random.default_rng(5).uniform(-1, 1, n).astype(dtype)
    dz = cu(np.zeros(n, dtype))
    pc.apply(cu(r), dz)
    want = reference.sor_apply(rp, ci, v, r, omega=1.9)
    assert rel_err(dz.cpu().numpy(), want) < (1e-12 if dtype == np.float64 else 1e-5)
    # M = 1 / (omega * diag(A)) in the matrix's precision (sor.cpp:29-32)
    assert np.array_equal(pc.factor().cpu().numpy(),
                          dtype(1) / (dtype(1.9) * v[_diag_pos(rp, ci)]))
    pc.close()
    A.close()


def _diag_pos(rp, ci):
    n = len(rp) - 1
    return np.array([rp[i] + int(np.nonzero(ci[rp[i]:rp[i + 1]] == i)[0][0]) for i in range(n)])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_sweep_forms_and_unaligned_rhs(handle, restatement, dtype):
    """Small systems take the single-CTA sweeps with the record ring, large
    ones the flag-synchronized sweeps; the ring sweeps give the same bits
    whether the right-hand side is bulk-copied (16-byte aligned) or read by
    plain loads (a view one element in), and agree with the oracle."""
    import torch
    from monolish_b200 import device as D
    for name, forms in (("poisson2d_40x37", (2, 2)), ("tiny_5", (2, 2)),
                        ("poisson2d_240", (0, 0))):
        rp, ci, v = MATS[name]
        v = v.astype(dtype)
        n = len(rp) - 1
        A = crs(handle, rp, ci, v)
        for kind in (SOR, ILU) + ((IC,) if name in SYM else ()):
            pc = D.Precond(A, kind, omega=1.9)
            assert pc.sweep_form() == forms, (name, kind)
            r = np.random.default_rng(9).uniform(-1, 1, n).astype(dtype)
            dz = cu(np.zeros(n, dtype))
            pc.apply(cu(r), dz)
            padded = cu(np.concatenate([np.zeros(1, dtype), r]))
            assert padded[1:].data_ptr() % 16 != 0
            dz2 = torch.zeros_like(dz)
            pc.apply(padded[1:], dz2)
            assert torch.equal(dz, dz2), (name, kind)
            want = restatement.precond_apply(rp, ci, v, kind, r, omega=1.9)
            assert rel_err(dz.cpu().numpy(), want) < (1e-12 if dtype == np.float64 else 1e-5)
            pc.close()
        A.close()


def test_known_answers(handle):
    """The reference's own sparse IC / ILU tests (test/equation/sparse_ic,
    sparse_ilu on test/test.mtx, test2.mtx): IC(0) / ILU(0) of a tridiagonal
    matrix is exact, so M^{-1} (A 1) = 1."""
    from monolish_b200 import device as D
    rp = np.array([0, 2, 5, 7], np.int32)
    ci = np.array([0, 1, 0, 1, 2, 1, 2], np.int32)
    cases = {"test.mtx": np.array([2, -1, -1, 2, -1, -1, 2.0]),
             "test2.mtx": np.array([2, 1, -1, 2, -1, 1, 2.0])}
    for name, v in cases.items():
        A = crs(handle, rp, ci, v)
        b = np.zeros(3)
        for i in range(3):
            b[i] = sum(v[j] for j in range(rp[i], rp[i + 1]))
        for kind in ((IC, ILU) if name == "test.mtx" else (ILU,)):
            pc = D.Precond(A, kind)
            dz = cu(np.zeros(3))
            pc.apply(cu(b), dz)
            assert np.allclose(dz.cpu().numpy(), 1.0, rtol=0, atol=1e-14)
            pc.close()
        A.close()


def test_zero_pivots(handle, restatement):
    from monolish_b200 import device as D
    # structural: row 1 has no diagonal
    rp = np.array([0, 2, 3, 5], np.int32)
    ci = np.array([0, 1, 0, 1, 2], np.int32)
    v = np.array([2.0, 1.0, 1.0, 1.0, 3.0])
    A = crs(handle, rp, ci, v)
    for kind in (IC, ILU):
        pc = D.Precond(A, kind)
        assert pc.zero_pivot() == (1, 1)
        pc.close()
    A.close()
    # numerical (ILU): [[1, 1], [1, 1]] -> u_11 = 0
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    v = np.array([1.0, 1.0, 1.0, 1.0])
    A = crs(handle, rp, ci, v)
    pc = D.Precond(A, ILU)
    assert pc.zero_pivot() == (1, 0)
    assert restatement.precond_factor(rp, ci, v, ILU)[1] == 1
    pc.close()
    # numerical (IC): not positive definite
    pc = D.Precond(A, IC)
    assert pc.zero_pivot() == (1, 0)
    pc.close()
    A.close()


def test_unsorted_rows_rejected(handle):
    from monolish_b200 import device as D
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([1, 0, 0, 1], np.int32)
    v = np.array([1.0, 4.0, 1.0, 4.0])
    A = crs(handle, rp, ci, v)
    for kind in (SOR, IC, ILU):
        with pytest.raises(_abi.MlshError) as e:
            D.Precond(A, kind)
        assert e.value.status == _abi.ERR_INVALID_CSR
    A.close()


def _pc_solve(handle, solver, kind, rp, ci, v, b, tol, maxiter, use_graph=True):
    from monolish_b200 import device as D
    n = len(rp) - 1
    A = crs(handle, rp, ci, v)
    pc = D.Precond(A, kind)
    dx = cu(np.zeros(n, v.dtype))
    fn = D.cg_solve_precond if solver == "cg" else D.bicgstab_solve_precond
    r = fn(A, pc, cu(b), dx, tol, maxiter, use_graph=use_graph)
    x = dx.cpu().numpy()
    pc.close()
    A.close()
    return r, x


CASES = [("cg", IC, "poisson2d"), ("cg", SOR, "poisson2d"), ("cg", ILU, "poisson3d"),
         ("bicgstab", ILU, "convdiff"), ("bicgstab", SOR, "convdiff"),
         ("bicgstab", IC, "poisson3d")]


def _system(which):
    if which == "poisson2d":
        rp, ci, v = W.poisson2d(64)[1:]
    elif which == "poisson3d":
        rp, ci, v = W.poisson3d(24)[1:]
    else:
        rp, ci, v = W.convdiff3d(20)[1:]
    n = len(rp) - 1
    xt = np.random.default_rng(2).uniform(-1, 1, n)
    b = np.zeros(n)
    for i in range(n):
        b[i] = np.dot(v[rp[i]:rp[i + 1]], xt[ci[rp[i]:rp[i + 1]]])
    return rp, ci, v, b


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("solver,kind,which", CASES)
def test_preconditioned_solves(handle, restatement, solver, kind, which, use_graph):
    rp, ci, v, b = _system(which)
    tol = 1e-10 * np.linalg.norm(b)
    r, x = _pc_solve(handle, solver, kind, rp, ci, v, b, tol, 2000, use_graph)
    fn = restatement.cg if solver == "cg" else restatement.bicgstab
    st, it, res, xo = fn(rp, ci, v, b, np.zeros(len(b)), tol, 2000, precond=kind)
    assert r.status == st
    assert abs(r.iters - it) <= 1, (r.iters, it)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
    assert restatement.true_relres(rp, ci, v, b, x) < 2e-10


def test_preconditioned_fp32(handle, restatement):
    rp, ci, v, b = _system("poisson2d")
    v32, b32 = v.astype(np.float32), b.astype(np.float32)
    tol = 1e-5 * float(np.linalg.norm(b))
    for solver, kind in (("cg", IC), ("bicgstab", ILU), ("cg", SOR)):
        r, x = _pc_solve(handle, solver, kind, rp, ci, v32, b32, tol, 2000)
        fn = restatement.cg if solver == "cg" else restatement.bicgstab
        st, it, _, _ = fn(rp, ci, v32, b32, np.zeros(len(b), np.float32), tol, 2000,
                          precond=kind)
        assert r.status == st == 0
        assert abs(r.iters - it) <= max(2, it // 10)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_sor_solver_matches_reference(handle, reference, dtype):
    from monolish_b200 import device as D
    rp, ci, v = W.poisson2d(24)[1:]
    v = v.astype(dtype)
    n = len(rp) - 1
    b = np.ones(n, dtype)
    tol = 1e-8 if dtype == np.float64 else 1e-4
    A = crs(handle, rp, ci, v)
    dx = cu(np.zeros(n, dtype))
    hist = np.zeros(5000)
    r = D.sor_solve(A, cu(b), dx, tol, 5000, omega=1.9, history=hist)
    st, it, res, xr, _ = reference.sor(rp, ci, v, b, np.zeros(n, dtype), tol, 5000, omega=1.9)
    assert r.status == st == 0
    assert abs(r.iters - it) <= (1 if dtype == np.float64 else max(2, it // 20))
    x = dx.cpu().numpy()
    assert rel_err(x, xr) < (1e-10 if dtype == np.float64 else 1e-3)
    assert abs(r.resid - res) <= 1e-6 * max(res, 1e-30) + (1e-12 if dtype == np.float64
                                                         else 1e-5)
    assert hist[r.iters - 1] < tol
    A.close()


def test_sor_solver_edges(handle, restatement):
    from monolish_b200 import device as D
    rp, ci, v = W.poisson2d(10)[1:]
    n = len(rp) - 1
    A = crs(handle, rp, ci, v)
    # maxiter reached
    dx = cu(np.zeros(n))
    r = D.sor_solve(A, cu(np.ones(n)), dx, 1e-30, 7)
    st, it, res, xo = restatement.sor(rp, ci, v, np.ones(n), np.zeros(n), 1e-30, 7)
    assert r.status == st == _abi.SOLVER_MAXITER and r.iters == it == 7
    assert rel_err(dx.cpu().numpy(), xo) < 1e-12
    # b = 0: ||r||/||b|| = 0 * inf is NaN at the first check
    dx = cu(np.zeros(n))
    r = D.sor_solve(A, cu(np.zeros(n)), dx, 1e-8, 100)
    st, it, _, _ = restatement.sor(rp, ci, v, np.zeros(n), np.zeros(n), 1e-8, 100)
    assert r.status == st == _abi.SOLVER_RESIDUAL_NAN and r.iters == it == 1
    # miniter honoured
    dx = cu(np.zeros(n))
    r = D.sor_solve(A, cu(np.ones(n)), dx, 10.0, 100, miniter=9)
    st, it, _, _ = restatement.sor(rp, ci, v, np.ones(n), np.zeros(n), 10.0, 100, miniter=9)
    assert r.status == st == 0 and r.iters == it == 9
    # another omega on the same plan rebuilds the sweep
    for om in (1.0, 1.5):
        dx = cu(np.zeros(n))
        r = D.sor_solve(A, cu(np.ones(n)), dx, 1e-10, 5000, omega=om)
        st, it, _, _ = restatement.sor(rp, ci, v, np.ones(n), np.zeros(n), 1e-10, 5000,
                                       omega=om)
        assert r.status == st and abs(r.iters - it) <= 1
    A.close()


def test_large_ic_cg_property(handle, restatement):
    """IC(0)-CG on a 3D Poisson 96^3 (884,736 rows, ~2,800 row blocks per
    sweep): converges with the oracle's iteration count and a true
    residual below the tolerance."""
    rp, ci, v = W.poisson3d(96)[1:]
    n = len(rp) - 1
    b = np.ones(n)
    tol = 1e-8 * np.linalg.norm(b)
    r, x = _pc_solve(handle, "cg", IC, rp, ci, v, b, tol, 5000)
    st, it, _, xo = restatement.cg(rp, ci, v, b, np.zeros(n), tol, 5000, precond=IC)
    assert r.status == st == 0
    assert abs(r.iters - it) <= 1
    assert restatement.true_relres(rp, ci, v, b, x) < 1e-8 * 1.01
