"""Solve server (mlsh_server_*): requests of mixed sizes, kinds and
precisions submitted while others run.

* every request against the oracle: status equal, iteration counts within
  +-2% (plain FP64; BiCGSTAB +-10% as in the batch tests), true relative
  residual below the requested tolerance x 10;
* each request's result is the same whether it runs alone on an idle
  server or inside the mix (bit-identical x, equal iteration count);
* admission is first-come first-served under the memory budget: with a
  budget of a few requests' footprint, later requests are admitted only
  after earlier ones complete, and all complete;
* a request larger than the whole budget completes with MLSH_ERR_OOM
  without disturbing the others; an empty system completes like the
  single-solve entry points.
"""
import threading
import time

import numpy as np
import pytest

from monolish_b200 import _abi
from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8
MAXITER = 20000


def _system(kind, n, seed):
    if kind == "cg":
        nx, ny = W.grid2d_for(int(n))
        _, rp, ci, v = W.vardiff2d(nx, ny, seed, 0)
    else:
        m = max(2, int(round(n ** (1.0 / 3.0))))
        _, rp, ci, v = W.convdiff3d(m, peclet=float(2 + seed % 7))
    return rp, ci, v


def _mix():
    """(kind, precision, n, seed): both ring classes (<= 4,096 rows on
    1-CTA clusters, <= 65,536 on 16-CTA clusters) and the worker lanes
    (larger, or mixed precision)."""
    out = []
    for k, n in enumerate([60, 400, 1500, 4000, 9000, 30000, 60000, 150000]):
        out.append(("cg", "fp64", n, 100 + k))
    for k, n in enumerate([300, 3000, 20000, 90000]):
        out.append(("bicgstab", "fp64", n, 200 + k))
    out.append(("cg", "mixed", 40000, 300))
    out.append(("bicgstab", "mixed", 70000, 301))
    return out


def _requests(restatement, mix):
    reqs = []
    for kind, prec, n, seed in mix:
        rp, ci, v = _system(kind, n, seed)
        xt = W.uniform_mt(len(rp) - 1, -1, 1, seed)
        b = restatement.spmv(rp, ci, v, xt)
        reqs.append(dict(kind=kind, precision=prec, rp=rp, ci=ci, v=v, b=b,
                         tol=REL_TOL * float(np.linalg.norm(b))))
    return reqs


def _submit(srv, q):
    return srv.submit(q["kind"], q["rp"], q["ci"], q["v"], q["b"], q["tol"], MAXITER,
                      precision=q["precision"], inner_tol=1e-4)


def _serve_all(reqs, budget=8 << 30, lanes=2, stagger=0.0):
    from monolish_b200 import device as D
    srv = D.Server(budget, lanes)
    ids = []
    for q in reqs:
        ids.append(_submit(srv, q))
        if stagger:
            time.sleep(stagger)
    res = [srv.wait(i) for i in ids]
    srv.close()
    return res


@pytest.fixture(scope="module")
def mix_results(cuda, restatement):
    reqs = _requests(restatement, _mix())
    # shuffled submission order, arriving while earlier ones run
    order = np.random.default_rng(5).permutation(len(reqs))
    res = _serve_all([reqs[i] for i in order], stagger=0.002)
    out = [None] * len(reqs)
    for j, i in enumerate(order):
        out[i] = res[j]
    return reqs, out


def test_serve_matches_oracle(mix_results, restatement):
    reqs, res = mix_results
    for q, r in zip(reqs, res):
        assert r.status == 0, (q["kind"], q["precision"], len(q["b"]), r.status)
        assert r.resid < q["tol"]
        rel = restatement.true_relres(q["rp"], q["ci"], q["v"], q["b"], r.x)
        assert rel < 10 * REL_TOL, (q["kind"], len(q["b"]), rel)
        if q["precision"] != "fp64":
            continue
        st, it, _, _ = getattr(restatement, q["kind"])(q["rp"], q["ci"], q["v"], q["b"],
                                                       np.zeros(len(q["b"])), q["tol"],
                                                       MAXITER)
        assert st == r.status
        slack = 0.02 if q["kind"] == "cg" else 0.10
        assert abs(r.iters - it) <= max(1, int(slack * it)), (q["kind"], len(q["b"]),
                                                              r.iters, it)


def test_serve_paths(mix_results):
    reqs, res = mix_results
    for q, r in zip(reqs, res):
        lane = q["precision"] != "fp64" or len(q["b"]) > 65536
        assert r.path == (1 if lane else 0)
        assert r.t_submit <= r.t_admit <= r.t_done


def test_serve_same_alone_and_in_mix(mix_results, restatement):
    reqs, res = mix_results
    for k in [1, 4, 6, 7, 9, 12]:  # both ring classes, lanes, BiCGSTAB, mixed
        alone = _serve_all([reqs[k]])[0]
        assert (alone.status, alone.iters) == (res[k].status, res[k].iters), k
        assert np.array_equal(alone.x, res[k].x), k


def test_serve_admission_fifo_under_budget(cuda, restatement):
    """Budget of about three requests: admission waits for completions,
    in arrival order, and every request completes."""
    from monolish_b200 import device as D
    reqs = _requests(restatement, [("cg", "fp64", 30000, 400 + k) for k in range(12)])
    nnz = int(reqs[0]["rp"][-1])
    n = len(reqs[0]["b"])
    foot = 4 * (n + 1) + 12 * nnz + 32 * n + 8192
    srv = D.Server(int(3.2 * foot), 1)
    ids = [_submit(srv, q) for q in reqs]
    res = [srv.wait(i) for i in ids]
    srv.close()
    assert all(r.status == 0 for r in res)
    admits = [r.t_admit for r in res]
    assert admits == sorted(admits)
    # at most three held at any admission (a request's memory is released
    # before its completion time is taken, and admission follows that)
    for j, rj in enumerate(res):
        held = sum(1 for r in res if r.t_admit <= rj.t_admit < r.t_done)
        assert held <= 3, (j, held)
    # and the budget did hold requests back
    assert any(res[j].t_admit > res[0].t_done for j in range(3, len(res)))


def test_serve_continuous_arrivals(cuda, restatement):
    """Requests submitted from another thread while the server runs."""
    from monolish_b200 import device as D
    reqs = _requests(restatement, [("cg", "fp64", int(n), 500 + k) for k, n in
                                   enumerate(np.geomspace(100, 20000, 24))])
    srv = D.Server(4 << 30, 1)
    ids = [None] * len(reqs)

    def producer():
        for k, q in enumerate(reqs):
            ids[k] = _submit(srv, q)
            time.sleep(0.001)

    t = threading.Thread(target=producer)
    t.start()
    t.join()
    res = [srv.wait(i) for i in ids]
    launches, lane_solves = srv.stats()
    srv.close()
    assert launches >= 1 and lane_solves == 0
    for q, r in zip(reqs, res):
        assert r.status == 0
        assert restatement.true_relres(q["rp"], q["ci"], q["v"], q["b"], r.x) < 10 * REL_TOL


def test_serve_oom_and_empty(cuda, restatement):
    from monolish_b200 import device as D
    big = _requests(restatement, [("cg", "fp64", 200000, 600)])[0]
    small = _requests(restatement, [("cg", "fp64", 1000, 601)])[0]
    srv = D.Server(16 << 20, 1)  # 16 MiB: the 200k-row system cannot fit
    i_big = _submit(srv, big)
    i_small = _submit(srv, small)
    i_empty = srv.submit("cg", np.zeros(1, np.int32), np.zeros(0, np.int32),
                         np.zeros(0), np.zeros(0), 1e-8, 100)
    r_big, r_small, r_empty = srv.wait(i_big), srv.wait(i_small), srv.wait(i_empty)
    srv.close()
    assert r_big.status == _abi.ERR_OOM
    assert r_small.status == 0
    assert (r_empty.status, r_empty.iters) == (0, 1)


def test_serve_result_released_once_read(cuda, restatement):
    from monolish_b200 import device as D
    q = _requests(restatement, [("cg", "fp64", 500, 700)])[0]
    srv = D.Server(1 << 30, 1)
    i = _submit(srv, q)
    r = srv.wait(i)
    assert r.status == 0
    res = _abi.RequestResult()
    assert srv.lib.mlsh_server_poll(srv.s, i, res) == _abi.ERR_INVALID_ARG
    srv.close()
