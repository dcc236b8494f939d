"""Matrix set-up on the GPU against the oracle: COO sort / merge, COO ->
CRS row pointers, CRS transposition and the transposed SpMV.

Integer results (orders, row pointers, indices) and gathered values are
bit-exact.  The transposed SpMV is bit-exact against the reference's serial
loop where each column has at most 8 entries (summed one after another in
row order, as the reference does) and within 1e-14 relative to the sum of
|a_ij x_i| elsewhere (segmented sums); FP32 within 1e-5 of that scale."""
import numpy as np
import pytest

from monolish_b200 import _abi
from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _random_coo(m, n, k, seed, dups=0):
    rng = np.random.default_rng(seed)
    lin = rng.choice(m * n, k, replace=False)
    row, col = (lin // n).astype(np.int32), (lin % n).astype(np.int32)
    val = rng.uniform(-1.0, 1.0, k)
    if dups:
        d = rng.integers(0, k, dups)
        row, col = np.concatenate([row, row[d]]), np.concatenate([col, col[d]])
        val = np.concatenate([val, rng.uniform(-1.0, 1.0, dups)])
        p = rng.permutation(len(row))
        row, col, val = row[p], col[p], val[p]
    return row, col, val


@pytest.mark.parametrize("m,n,k,dups", [(400, 300, 3000, 0), (400, 300, 3000, 600),
                                        (1, 1, 1, 0), (70000, 300, 200000, 5000),
                                        (5000, 5000000, 300000, 1000)])
@pytest.mark.parametrize("merge", [True, False])
def test_coo_sort_matches_oracle(handle, restatement, m, n, k, dups, merge):
    from monolish_b200 import device as D
    row, col, val = _random_coo(m, n, k, seed=m + k, dups=dups)
    dr, dc, dv = _dev(row), _dev(col), _dev(val)
    cnt = D.coo_sort(handle, m, n, dr, dc, dv, merge=merge)
    er, ec, ev = restatement.coo_sort(row, col, val, merge)
    assert cnt == len(er)
    assert np.array_equal(dr.cpu().numpy()[:cnt], er)
    assert np.array_equal(dc.cpu().numpy()[:cnt], ec)
    assert np.array_equal(dv.cpu().numpy()[:cnt], ev)


def test_coo_sort_golden_and_float(handle, restatement):
    import torch
    from monolish_b200 import device as D
    g = np.load(__file__.replace("test_gpu_setup.py", "golden/setup.npz"))
    dr, dc, dv = _dev(g["coo_row"]), _dev(g["coo_col"]), _dev(g["coo_val"])
    cnt = D.coo_sort(handle, 400, 300, dr, dc, dv, merge=True)
    assert np.array_equal(dr.cpu().numpy()[:cnt], g["sorted_row"])
    assert np.array_equal(dc.cpu().numpy()[:cnt], g["sorted_col"])
    assert np.array_equal(dv.cpu().numpy()[:cnt], g["sorted_val"])
    rp = D.coo_to_csr(handle, 400, dr, cnt)
    assert np.array_equal(rp.cpu().numpy(), g["rowptr"])
    dr, dc = _dev(g["dup_row"]), _dev(g["dup_col"])
    dv = _dev(g["dup_val"].astype(np.float32))
    cnt = D.coo_sort(handle, 400, 300, dr, dc, dv, merge=True)
    assert np.array_equal(dr.cpu().numpy()[:cnt], g["dup_merged_row"])
    assert np.array_equal(dc.cpu().numpy()[:cnt], g["dup_merged_col"])
    er, ec, ev = restatement.coo_sort(g["dup_row"], g["dup_col"], g["dup_val"], True)
    assert dv.dtype == torch.float32
    assert np.array_equal(dv.cpu().numpy()[:cnt], ev.astype(np.float32))


def test_coo_errors(handle):
    from monolish_b200 import device as D
    row, col, val = _random_coo(50, 40, 100, seed=1)
    col[7] = 40  # out of range
    with pytest.raises(_abi.MlshError) as e:
        D.coo_sort(handle, 50, 40, _dev(row), _dev(col), _dev(val))
    assert e.value.status == _abi.ERR_INVALID_ARG
    rows = _dev(np.array([0, 2, 1], np.int32))  # not row-sorted
    with pytest.raises(_abi.MlshError) as e:
        D.coo_to_csr(handle, 3, rows)
    assert e.value.status == _abi.ERR_INVALID_CSR


def test_coo_to_csr_empty_rows(handle, restatement):
    from monolish_b200 import device as D
    row = np.array([2, 2, 5, 5, 5, 9], np.int32)
    rp = D.coo_to_csr(handle, 12, _dev(row)).cpu().numpy()
    assert np.array_equal(rp, restatement.coo_rowptr(12, row))
    rp = D.coo_to_csr(handle, 4, _dev(np.zeros(0, np.int32)), 0).cpu().numpy()
    assert np.array_equal(rp, np.zeros(5, np.int32))


def _matrices():
    yield "poisson3d_20", W.poisson3d(20)[1:], 8000
    n, rp, ci, v = W.zipf(30000, seed=5, maxlen=4000, ncols=20000)
    yield "zipf_rect", (rp, ci, v), 20000
    rp = np.array([0, 0, 3, 3, 5, 5], np.int32)  # empty rows, empty columns
    yield "ragged", (rp, np.array([1, 4, 6, 0, 6], np.int32), np.arange(1.0, 6.0)), 9


@pytest.mark.parametrize("case", list(_matrices()), ids=lambda c: c[0])
def test_csr_transpose_matches_oracle(handle, restatement, case):
    from monolish_b200 import device as D
    _, (rp, ci, v), n_cols = case
    n_rows = len(rp) - 1
    rp_t, ci_t, v_t = D.csr_transpose(handle, n_rows, n_cols, _dev(rp), _dev(ci), _dev(v))
    e_rp, e_ci, e_v = restatement.csr_transpose(rp, ci, v, n_cols)
    assert np.array_equal(rp_t.cpu().numpy(), e_rp)
    assert np.array_equal(ci_t.cpu().numpy(), e_ci)
    assert np.array_equal(v_t.cpu().numpy(), e_v)


@pytest.mark.parametrize("case", list(_matrices()), ids=lambda c: c[0])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spmv_transpose_matches_oracle(handle, restatement, case, dtype):
    import torch
    from monolish_b200 import device as D
    _, (rp, ci, v), n_cols = case
    n_rows = len(rp) - 1
    v = v.astype(dtype)
    x = W.uniform_mt(n_rows, -1.0, 1.0, 7).astype(dtype)
    A = D.Crs(handle, n_rows, n_cols, rp, ci, v)
    dx = _dev(x)
    dy = torch.full((n_cols,), float("nan"), dtype=dx.dtype, device="cuda")
    A.matvec_t(dx, dy)
    y = dy.cpu().numpy()
    e = restatement.spmv_t(rp, ci, v, x, n_cols)
    counts = np.bincount(ci, minlength=n_cols)
    short = counts <= 8
    if dtype == np.float64:
        assert np.array_equal(y[short], e[short])
    scale = np.abs(restatement.spmv_t(rp, ci, np.abs(v), np.abs(x), n_cols)).astype(np.float64)
    tol = 1e-14 if dtype == np.float64 else 1e-5
    assert np.all(np.abs(y.astype(np.float64) - e) <= tol * np.maximum(scale, 1e-300) + 1e-300)
    # alpha / beta, and a values change refreshing the cached transpose
    y0 = W.uniform_mt(n_cols, -1.0, 1.0, 8).astype(dtype)
    dy = _dev(y0)
    A.matvec_t(dx, dy, alpha=0.5, beta=2.0)
    ref = 0.5 * e.astype(np.float64) + 2.0 * y0.astype(np.float64)
    assert np.all(np.abs(dy.cpu().numpy() - ref) <= 2 * tol * (scale + np.abs(ref)) + 1e-300)
    A.d_val.mul_(3.0)
    A.values_changed()
    A.matvec_t(dx, dy)
    e3 = restatement.spmv_t(rp, ci, (v * 3).astype(dtype), x, n_cols)
    assert np.all(np.abs(dy.cpu().numpy().astype(np.float64) - e3)
                  <= 3 * tol * np.maximum(scale, 1e-300) + 1e-300)
    A.close()


def test_spmv_transpose_golden(handle):
    import torch
    from monolish_b200 import device as D
    g = np.load(__file__.replace("test_gpu_setup.py", "golden/setup.npz"))
    rp, ci, v = g["zipf_rp"], g["zipf_ci"], g["zipf_v"]
    A = D.Crs(handle, len(rp) - 1, 1000, rp, ci, v)
    dy = torch.zeros(1000, dtype=torch.float64, device="cuda")
    A.matvec_t(_dev(g["zipf_x"]), dy)
    y = dy.cpu().numpy()
    counts = np.bincount(ci, minlength=1000)
    assert np.array_equal(y[counts <= 8], g["zipf_yt"][counts <= 8])
    assert np.allclose(y, g["zipf_yt"], rtol=1e-13, atol=1e-13)
    A.close()


def test_large_sort_properties(handle):
    """Multi-pass radix sort at 2^24 + 3 entries: (row, col) order, a
    permutation of the input, and no entry lost."""
    from monolish_b200 import device as D
    rng = np.random.default_rng(99)
    k = (1 << 24) + 3
    row = rng.integers(0, 1 << 22, k, dtype=np.int32)
    col = rng.integers(0, 1 << 21, k, dtype=np.int32)
    val = np.arange(k, dtype=np.float64)  # the value records the input position
    dr, dc, dv = _dev(row), _dev(col), _dev(val)
    cnt = D.coo_sort(handle, 1 << 22, 1 << 21, dr, dc, dv, merge=False)
    assert cnt == k
    order = np.lexsort((np.arange(k), col, row))
    assert np.array_equal(dv.cpu().numpy(), val[order])
    assert np.array_equal(dr.cpu().numpy(), row[order])
    assert np.array_equal(dc.cpu().numpy(), col[order])
