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


def test_setup_routines_match_reference_golden(restatement):
    """Transposed SpMV, COO sort/merge and the COO -> CRS row pointer of the
    restatement against the reference's blas::matvec_T, COO::sort and
    CRS(COO&) outputs."""
    g = golden("setup")
    yt = restatement.spmv_t(g["zipf_rp"], g["zipf_ci"], g["zipf_v"], g["zipf_x"], 1000)
    assert np.array_equal(yt, g["zipf_yt"])  # same serial loop: identical bits
    n, rp, ci, v = W.poisson2d(16)
    assert np.array_equal(restatement.spmv_t(rp, ci, v, g["pois_x"], n), g["pois_yt"])
    sr, sc, sv = restatement.coo_sort(g["coo_row"], g["coo_col"], g["coo_val"], True)
    assert np.array_equal(sr, g["sorted_row"]) and np.array_equal(sc, g["sorted_col"])
    assert np.array_equal(sv, g["sorted_val"])
    assert np.array_equal(restatement.coo_rowptr(400, sr), g["rowptr"])
    dr, dc, _ = restatement.coo_sort(g["dup_row"], g["dup_col"], g["dup_val"], True)
    assert np.array_equal(dr, g["dup_merged_row"]) and np.array_equal(dc, g["dup_merged_col"])
    nr, nc, _ = restatement.coo_sort(g["dup_row"], g["dup_col"], g["dup_val"], False)
    assert np.array_equal(nr, g["dup_all_row"]) and np.array_equal(nc, g["dup_all_col"])
    # the restatement's transpose is scipy's CSR transpose with sorted indices
    import scipy.sparse as sp
    rp_t, ci_t, v_t = restatement.csr_transpose(g["zipf_rp"], g["zipf_ci"], g["zipf_v"], 1000)
    At = sp.csr_matrix((g["zipf_v"], g["zipf_ci"], g["zipf_rp"]), shape=(1500, 1000)).T.tocsr()
    At.sort_indices()
    assert np.array_equal(rp_t, At.indptr) and np.array_equal(ci_t, At.indices)
    assert np.array_equal(v_t, At.data)


def test_setup_routines_match_reference_live(restatement, reference):
    n, rp, ci, v = W.zipf(5000, seed=9, maxlen=3000, ncols=3500)
    x = W.uniform_mt(n, -1.0, 1.0, 41)
    assert np.array_equal(restatement.spmv_t(rp, ci, v, x, 3500),
                          reference.spmv_t(rp, ci, v, x, 3500))
    rng = np.random.default_rng(42)
    lin = rng.choice(900 * 700, 20000, replace=False)
    row, col = (lin // 700).astype(np.int32), (lin % 700).astype(np.int32)
    val = rng.uniform(-1, 1, 20000)
    a = restatement.coo_sort(row, col, val, True)
    b = reference.coo_sort(900, 700, row, col, val, True)
    assert all(np.array_equal(p, q) for p, q in zip(a, b))
    assert np.array_equal(restatement.coo_rowptr(900, a[0]),
                          reference.coo_rowptr(900, 700, *b))
