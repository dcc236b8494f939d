"""Regenerate the golden fixtures in this directory from the reference.

The fixtures pin the oracle (and through it the CUDA path) to the
reference's own CPU implementation: each case runs the reference monolish
CPU library built from the reference sources (oracle/_ref, see
oracle/Makefile) through its public API -- CRS from raw arrays,
blas::matvec/dot/nrm2/axpy/xpay/axpyz, equation::CG / BiCGSTAB::solve with
Jacobi or none -- on seeded inputs from monolish_b200/workloads.py, and
stores inputs and outputs.

    python tests/golden/make_golden.py      # needs oracle/_ref built

Cases (all small, so the CPU restatement replays them in seconds):
  tridiag3     the reference's own test matrix test/test.mtx (3x3
               tridiagonal 2,-1); b = A*ones, x0 ~ U(0,1) from
               mt19937(1234) as in test/test_utils.hpp:21; CG and
               BiCGSTAB, none/Jacobi, double (tol 1e-8) and float (1e-4).
  poisson16    2D 5-point 16x16, x_true ~ U[-1,1] seed 0, x0 = 0,
               tol = 1e-10*||b||, Jacobi CG and BiCGSTAB.
  poisson128   the 128x128 Jacobi-CG workload (n = 16,384).
  convdiff10   3D upwind convection-diffusion 10^3, Peclet 10, Jacobi
               BiCGSTAB, tol 1e-10*||b||.
  zipf_spmv    SpMV on an 8,000-row Zipf(2) matrix (lengths up to 8,000;
               four rows exceed one 1,792-nonzero SpMV tile), double and
               float.
  blas1        dot/nrm2/axpy/xpay/axpyz on n = 1,000.
  setup        blas::matvec_T on a 1,500 x 1,000 Zipf(2) matrix and on
               the 16x16 Poisson matrix; COO::sort(merge) of a shuffled
               COO (400 x 300, 3,000 distinct entries) with the CRS(COO&)
               row pointer; the (row, col) sequence COO::sort leaves when
               600 duplicates are added (their kept values depend on the
               reference's quicksort order and are not stored).
  precond      equation::SOR (omega 1.9): create_precond + apply_precond on
               a 3D 7-point 8^3 Poisson matrix and on a 500-row random
               nonsymmetric matrix (sorted rows), double and float;
               SOR::solve on the 16x16 Poisson matrix (b = ones, tol 1e-8 /
               1e-4); CG and BiCGSTAB preconditioned by SOR on poisson16.

  fullsize     the measured configurations at full size, as summaries:
               SpMV on the 3D 7-point 256^3 Laplacian and the n = 4,194,304
               Zipf(2) matrix (FP64 and FP32): sum, sum of |y| and 4,096
               sampled rows; Jacobi-BiCGSTAB on the 160^3 convection-
               diffusion system (status, iterations, residuals); Jacobi-CG on
               each of the 2,048 batch systems (status, iterations).

    python tests/golden/make_golden.py setup     # that case only
    python tests/golden/make_golden.py precond   # that case only
    python tests/golden/make_golden.py fullsize  # that case only (minutes)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from monolish_b200 import workloads as W  # noqa: E402


def tridiag3():
    rp = np.array([0, 2, 5, 7], np.int32)
    ci = np.array([0, 1, 0, 1, 2, 1, 2], np.int32)
    v = np.array([2, -1, -1, 2, -1, -1, 2], np.float64)
    return 3, rp, ci, v


def setup_case(ref):
    out = {}
    n, rp, ci, v = W.zipf(1500, seed=3, maxlen=600, ncols=1000)
    x = W.uniform_mt(n, -1.0, 1.0, 31)
    out.update(zipf_rp=rp, zipf_ci=ci, zipf_v=v, zipf_x=x,
               zipf_yt=ref.spmv_t(rp, ci, v, x, 1000))
    n, rp, ci, v = W.poisson2d(16)
    x = W.uniform_mt(n, -1.0, 1.0, 32)
    out.update(pois_x=x, pois_yt=ref.spmv_t(rp, ci, v, x, n))
    rng = np.random.default_rng(33)
    m, k, cols = 400, 3000, 300
    lin = rng.choice(m * cols, k, replace=False)
    row, col = (lin // cols).astype(np.int32), (lin % cols).astype(np.int32)
    val = rng.uniform(-1.0, 1.0, k)
    sr, sc, sv = ref.coo_sort(m, cols, row, col, val, True)
    out.update(coo_row=row, coo_col=col, coo_val=val, sorted_row=sr, sorted_col=sc,
               sorted_val=sv, rowptr=ref.coo_rowptr(m, cols, sr, sc, sv))
    d = rng.integers(0, k, 600)
    row2, col2 = np.concatenate([row, row[d]]), np.concatenate([col, col[d]])
    val2 = np.concatenate([val, rng.uniform(-1.0, 1.0, 600)])
    dr, dc, _ = ref.coo_sort(m, cols, row2, col2, val2, True)
    nr, nc, _ = ref.coo_sort(m, cols, row2, col2, val2, False)
    out.update(dup_row=row2, dup_col=col2, dup_val=val2, dup_merged_row=dr, dup_merged_col=dc,
               dup_all_row=nr, dup_all_col=nc)
    return out


def random_sorted(n, per_row, seed):
    """Diagonally dominant nonsymmetric CRS with sorted rows."""
    rng = np.random.default_rng(seed)
    rp, ci, v = [0], [], []
    for i in range(n):
        cols = np.unique(np.append(rng.choice(n, per_row, replace=False), i))
        vals = rng.uniform(-1, 1, len(cols))
        vals[cols == i] = np.abs(vals).sum() + 1.0
        ci.extend(cols.tolist())
        v.extend(vals.tolist())
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v)


def precond_case(ref):
    out = {}
    _, rp, ci, v = W.poisson3d(8)
    rr, rc, rv = random_sorted(500, 6, 5)
    for tag, (a, b, c) in (("p3", (rp, ci, v)), ("rnd", (rr, rc, rv))):
        n = len(a) - 1
        r = W.uniform_mt(n, -1.0, 1.0, 51)
        out[f"{tag}_rp"], out[f"{tag}_ci"], out[f"{tag}_v"], out[f"{tag}_r"] = a, b, c, r
        out[f"{tag}_z_d"] = ref.sor_apply(a, b, c, r, omega=1.9)
        out[f"{tag}_z_s"] = ref.sor_apply(a, b, c.astype(np.float32), r.astype(np.float32),
                                          omega=1.9)
    n, rp, ci, v = W.poisson2d(16)
    b = np.ones(n)
    for sfx, dt, tol in (("d", np.float64, 1e-8), ("s", np.float32, 1e-4)):
        st, it, res, x, _ = ref.sor(rp, ci, v.astype(dt), b.astype(dt), np.zeros(n, dt), tol,
                                    5000, omega=1.9)
        out[f"sor_{sfx}"] = np.array([st, it, res])
        out[f"sor_{sfx}_x"] = x
    for solver in ("cg", "bicgstab"):
        st, it, res, x, _ = getattr(ref, solver)(rp, ci, v, b, np.zeros(n), 1e-8, 2000,
                                                 precond=2)
        out[f"{solver}_sor"] = np.array([st, it, res])
        out[f"{solver}_sor_x"] = x
    return out


def sample_rows(n, count=4096):
    return np.linspace(0, n - 1, count).round().astype(np.int64)


def fullsize_case(ref):
    """The measured configurations at full size.  Only small summaries are
    stored (the inputs are regenerated from their seeds by the tests):
    SpMV outputs as their sum, sum of |y| and 4,096 evenly spaced rows;
    solves as (status, iterations, final residual) per system."""
    ref.set_threads(os.cpu_count() or 1)
    out = {}
    # C2a / C2b SpMV, FP64 and FP32 (x as in the bench: U[-1,1], seed 1)
    for tag, gen in (("lap256", lambda: W.poisson3d(256)),
                     ("zipf4m", lambda: W.zipf(4194304, seed=1))):
        n, rp, ci, v = gen()
        x = W.uniform_fast(n, -1.0, 1.0, 1)
        rows = sample_rows(n)
        for sfx, dt in (("d", np.float64), ("s", np.float32)):
            y = ref.spmv(rp, ci, v.astype(dt), x.astype(dt))[0].astype(np.float64)
            out[f"{tag}_{sfx}_rows"] = rows
            out[f"{tag}_{sfx}_y"] = y[rows]
            out[f"{tag}_{sfx}_sum"] = np.array([y.sum(), np.abs(y).sum()])
        del rp, ci, v, x
        print(tag, "done", flush=True)
    # C3: Jacobi-BiCGSTAB on the 160^3 convection-diffusion system, FP64
    n, rp, ci, v = W.convdiff3d(160, peclet=10.0)
    xt = W.uniform_mt(n, -1.0, 1.0, 2)
    b = ref.spmv(rp, ci, v, xt)[0]
    nb = float(np.linalg.norm(b))
    st, it, res, x, sec = ref.bicgstab(rp, ci, v, b, np.zeros(n), 1e-10 * nb, 20000, precond=1)
    r = b - ref.spmv(rp, ci, v, x)[0]
    out["convdiff160_bicgstab"] = np.array([st, it, res, np.linalg.norm(r) / nb, nb])
    out["convdiff160_b_sum"] = np.array([b.sum(), np.abs(b).sum()])
    print("convdiff160", st, it, np.linalg.norm(r) / nb, f"{sec:.1f}s", flush=True)
    # C4: the 2,048-system diffusion batch, Jacobi-CG to 1e-8 (x_true seed 3 + k)
    systems = W.diffusion_batch(2048, seed=3)
    rec = np.zeros((len(systems), 4))
    for k, (rp, ci, v) in enumerate(systems):
        nk = len(rp) - 1
        b = ref.spmv(rp, ci, v, W.uniform_mt(nk, -1.0, 1.0, 3 + k))[0]
        nb = float(np.linalg.norm(b))
        st, it, res, x, _ = ref.cg(rp, ci, v, b, np.zeros(nk), 1e-8 * nb, 20000, precond=1)
        rec[k] = (st, it, res, nb)
    out["batch2048_cg"] = rec
    print("batch2048 iters", int(rec[:, 1].sum()), flush=True)
    return out


def main(only=None):
    ref = oracle.Reference()
    out = {}
    if only in ("setup", "precond", "fullsize"):
        out[only] = {"setup": setup_case, "precond": precond_case,
                     "fullsize": fullsize_case}[only](ref)
        for name, case in out.items():
            path = os.path.join(HERE, f"{name}.npz")
            np.savez_compressed(path, **case)
            print("wrote", path, os.path.getsize(path), "bytes")
        return

    # ---- tridiag3 (reference test/test.mtx) ----
    n, rp, ci, v = tridiag3()
    ones = np.ones(n)
    b = ref.spmv(rp, ci, v, ones)[0]
    x0 = ref.random_vector(n, 0.0, 1.0, 1234)
    case = dict(rp=rp, ci=ci, v=v, b=b, x0=x0)
    for solver in ("cg", "bicgstab"):
        for pre in (0, 1):
            st, it, res, x, _ = getattr(ref, solver)(rp, ci, v, b, x0, 1e-8, 10000, precond=pre)
            case[f"{solver}_p{pre}_d"] = np.array([st, it, res])
            case[f"{solver}_p{pre}_d_x"] = x
            vf, bf, x0f = v.astype(np.float32), b.astype(np.float32), x0.astype(np.float32)
            st, it, res, x, _ = getattr(ref, solver)(rp, ci, vf, bf, x0f, 1e-4, 10000,
                                                     precond=pre)
            case[f"{solver}_p{pre}_s"] = np.array([st, it, res])
            case[f"{solver}_p{pre}_s_x"] = x
    out["tridiag3"] = case

    # ---- Poisson solves ----
    for name, m in (("poisson16", 16), ("poisson128", 128)):
        n, rp, ci, v = W.poisson2d(m)
        xt = W.uniform_mt(n, -1.0, 1.0, 0)
        b = ref.spmv(rp, ci, v, xt)[0]
        tol = 1e-10 * np.linalg.norm(b)
        case = dict(rp=rp, ci=ci, v=v, b=b, tol=np.array(tol))
        solvers = ("cg", "bicgstab") if m == 16 else ("cg",)
        for solver in solvers:
            st, it, res, x, _ = getattr(ref, solver)(rp, ci, v, b, np.zeros(n), tol, 2000,
                                                     precond=1)
            case[f"{solver}"] = np.array([st, it, res])
            case[f"{solver}_x"] = x
        out[name] = case

    # ---- convection-diffusion BiCGSTAB ----
    n, rp, ci, v = W.convdiff3d(10, peclet=10.0)
    xt = W.uniform_mt(n, -1.0, 1.0, 2)
    b = ref.spmv(rp, ci, v, xt)[0]
    tol = 1e-10 * np.linalg.norm(b)
    st, it, res, x, _ = ref.bicgstab(rp, ci, v, b, np.zeros(n), tol, 2000, precond=1)
    out["convdiff10"] = dict(rp=rp, ci=ci, v=v, b=b, tol=np.array(tol),
                             bicgstab=np.array([st, it, res]), bicgstab_x=x)

    # ---- Zipf SpMV (long rows split across tiles) ----
    n, rp, ci, v = W.zipf(8000, seed=7, maxlen=8000)
    x = W.uniform_mt(n, -1.0, 1.0, 11)
    y = ref.spmv(rp, ci, v, x)[0]
    ys = ref.spmv(rp, ci, v.astype(np.float32), x.astype(np.float32))[0]
    out["zipf_spmv"] = dict(rp=rp, ci=ci, v=v, x=x, y=y, y_s=ys)

    # ---- vector BLAS ----
    a = W.uniform_mt(1000, -1.0, 1.0, 21)
    c = W.uniform_mt(1000, -1.0, 1.0, 22)
    out["blas1"] = dict(x=a, y=c, dot=np.array(ref.dot(a, c)), nrm2=np.array(ref.nrm2(a)),
                        axpy=ref.axpy(0.75, a, c), xpay=ref.xpay(0.75, a, c),
                        axpyz=ref.axpyz(0.75, a, c))

    out["setup"] = setup_case(ref)
    out["precond"] = precond_case(ref)

    for name, case in out.items():
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **case)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
