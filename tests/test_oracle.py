"""The oracle, pinned: the C restatement against the committed golden
fixtures (made from the reference build) and, where the reference CPU build
is present, against the reference itself.  CPU only."""
import os

import numpy as np
import pytest

from monolish_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def test_spmv_matches_reference_golden_bitwise(restatement):
    g = golden("zipf_spmv")
    rp, ci, v, x = g["rp"], g["ci"], g["v"], g["x"]
    # same row loop, same order, no FMA: identical bits
    assert np.array_equal(restatement.spmv(rp, ci, v, x), g["y"])
    ys = restatement.spmv(rp, ci, v.astype(np.float32), x.astype(np.float32))
    assert np.array_equal(ys, g["y_s"])


def test_blas1_matches_reference_golden(restatement):
    g = golden("blas1")
    x, y = g["x"], g["y"]
    # dot goes through an external CBLAS in the reference: order differs
    assert abs(restatement.dot(x, y) - float(g["dot"])) <= 1e-14 * np.sum(np.abs(x * y))
    assert abs(restatement.nrm2(x) - float(g["nrm2"])) <= 1e-14 * float(g["nrm2"])
    np.testing.assert_allclose(0.75 * x + y, g["axpy"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(x + 0.75 * y, g["xpay"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(0.75 * x + y, g["axpyz"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("solver", ["cg", "bicgstab"])
@pytest.mark.parametrize("pre", [0, 1])
@pytest.mark.parametrize("prec", ["d", "s"])
def test_tridiag3_solvers_match_reference_golden(restatement, solver, pre, prec):
    g = golden("tridiag3")
    dt = np.float64 if prec == "d" else np.float32
    tol = 1e-8 if prec == "d" else 1e-4
    st, it, res, x = getattr(restatement, solver)(
        g["rp"], g["ci"], g["v"].astype(dt), g["b"].astype(dt), g["x0"].astype(dt), tol, 10000,
        precond=pre)
    gst, git, gres = g[f"{solver}_p{pre}_{prec}"]
    assert st == int(gst) and it == int(git)
    np.testing.assert_allclose(x, g[f"{solver}_p{pre}_{prec}_x"], rtol=10 * tol, atol=10 * tol)
    # the reference's own answer check (equation_kernel.hpp: x vs ones at tol*10)
    np.testing.assert_allclose(x, np.ones(3), rtol=10 * tol)


@pytest.mark.parametrize("name,solver", [("poisson16", "cg"), ("poisson16", "bicgstab"),
                                         ("poisson128", "cg"), ("convdiff10", "bicgstab")])
def test_solves_match_reference_golden(restatement, name, solver):
    g = golden(name)
    rp, ci, v, b = g["rp"], g["ci"], g["v"], g["b"]
    tol = float(g["tol"])
    st, it, res, x = getattr(restatement, solver)(rp, ci, v, b, np.zeros_like(b), tol, 2000)
    gst, git, gres = g[solver]
    assert st == int(gst) == 0
    # +-2% iterations; BiCGSTAB on a symmetric matrix (poisson16) is the one
    # rounding-sensitive case: its iterates depend on the last bits of the
    # dots/axpys, which the reference takes from OpenBLAS's FMA kernels, so
    # there the bound is +-10%.
    slack = 0.10 if (solver == "bicgstab" and name.startswith("poisson")) else 0.02
    assert abs(it - int(git)) <= max(1, int(slack * git))
    gx = g[f"{solver}_x"]
    assert np.linalg.norm(x - gx) <= 1e-8 * np.linalg.norm(gx)
    assert restatement.true_relres(rp, ci, v, b, x) < 2e-10


def test_poisson128_is_the_reference_workload(restatement):
    """382 Jacobi-CG iterations to 1e-10 relative, as the reference runs it."""
    g = golden("poisson128")
    n, rp, ci, v = W.poisson2d(128)
    assert np.array_equal(rp, g["rp"]) and np.array_equal(ci, g["ci"])
    assert np.array_equal(v, g["v"])
    assert int(g["cg"][1]) == 382


def test_generators_match_reference(reference):
    n, rp, ci, v = W.poisson2d(37, 23)
    _, rp2, ci2, v2 = reference.laplacian_2d5p(37, 23)
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
    assert np.array_equal(W.uniform_mt(5000, -1, 1, 0), reference.random_vector(5000, -1, 1, 0))


def test_restatement_matches_reference_live(restatement, reference):
    n, rp, ci, v = W.zipf(2500, seed=3, maxlen=4000)
    x = W.uniform_mt(n, -1.0, 1.0, 5)
    assert np.array_equal(restatement.spmv(rp, ci, v, x), reference.spmv(rp, ci, v, x)[0])
    n, rp, ci, v = W.convdiff3d(8, peclet=3.0)
    b = restatement.spmv(rp, ci, v, W.uniform_mt(n, -1, 1, 2))
    tol = 1e-10 * np.linalg.norm(b)
    for solver in ("cg", "bicgstab"):
        if solver == "cg":
            n2, rp2, ci2, v2 = W.vardiff2d(20, 17, 3, 0)
            b2 = restatement.spmv(rp2, ci2, v2, W.uniform_mt(n2, -1, 1, 2))
            args = (rp2, ci2, v2, b2, np.zeros(n2), 1e-10 * np.linalg.norm(b2), 3000)
        else:
            args = (rp, ci, v, b, np.zeros(n), tol, 3000)
        st1, it1, r1, x1 = getattr(restatement, solver)(*args)
        st2, it2, r2, x2, _ = getattr(reference, solver)(*args)
        assert st1 == st2 == 0
        assert abs(it1 - it2) <= max(1, int(0.02 * it2))
        assert np.linalg.norm(x1 - x2) <= 1e-8 * np.linalg.norm(x2)


def test_status_codes_match_reference(restatement, reference):
    n, rp, ci, v = W.poisson2d(8)
    b = np.zeros(n)
    # b = 0, x0 = 0: CG divides 0/0 -> NaN residual; BiCGSTAB breaks down (rho = 0)
    for solver in ("cg", "bicgstab"):
        a = getattr(restatement, solver)(rp, ci, v, b, np.zeros(n), 1e-10, 100)
        r = getattr(reference, solver)(rp, ci, v, b, np.zeros(n), 1e-10, 100)
        assert a[0] == r[0] and a[1] == r[1]
    # maxiter
    b = restatement.spmv(rp, ci, v, np.ones(n))
    a = restatement.cg(rp, ci, v, b, np.zeros(n), 1e-30, 5)
    r = reference.cg(rp, ci, v, b, np.zeros(n), 1e-30, 5)
    assert a[0] == r[0] == -2 and a[1] == r[1] == 5
