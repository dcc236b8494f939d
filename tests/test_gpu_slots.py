"""The offset-slot layout of FP32 plans (mlsh_csr_plan_set_layout): the
same y as the CRS kernel, bit for bit, on the matrices it takes (stencils,
boundary rows with missing neighbours, a last slice cut short, the unit
diagonal of a Jacobi-scaled copy, alpha/beta), and a clean refusal on the
ones it does not (rows longer than 8 entries, unsorted rows)."""
import numpy as np
import pytest

from monolish_b200 import workloads as W

pytestmark = pytest.mark.gpu


def spmv_both(handle, n, rp, ci, v, x, alpha=1.0, beta=0.0, y0=None):
    import torch
    from monolish_b200.device import Crs
    A = Crs(handle, n, n, rp, ci, v)
    dx = torch.from_numpy(x).cuda()
    out = {}
    for layout in (0, 1):
        applied = A.set_layout(layout)
        dy = (torch.from_numpy(y0.copy()).cuda() if y0 is not None
              else torch.full((n,), float("nan"), dtype=dx.dtype, device="cuda"))
        A.matvec(dx, dy, alpha, beta)
        handle.sync()
        out[layout] = (applied, dy.cpu().numpy())
    A.close()
    return out


@pytest.mark.parametrize("case", ["convdiff37", "poisson2d_77x53", "poisson3d_20"])
def test_slots_bitwise_equal_to_crs(handle, restatement, case):
    if case == "convdiff37":
        n, rp, ci, v = W.convdiff3d(37, peclet=10.0)  # 50,653 rows: last slice cut short
    elif case == "poisson2d_77x53":
        n, rp, ci, v = W.poisson2d(77, 53)
    else:
        n, rp, ci, v = W.poisson3d(20)
    v = v.astype(np.float32)
    x = W.uniform_mt(n, -1, 1, 5).astype(np.float32)
    out = spmv_both(handle, n, rp, ci, v, x)
    assert out[0][0] and out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[1][1], restatement.spmv(rp, ci, v, x))


def test_slots_unit_diagonal(handle, restatement):
    """A D^-1 rounded to FP32 has an exact unit diagonal: the layout stores
    no diagonal and adds x_i in its place."""
    n, rp, ci, v = W.convdiff3d(30, peclet=3.0)
    rows = np.repeat(np.arange(n), np.diff(rp))
    d = v[ci == rows]
    v32 = (v * (1.0 / d)[ci]).astype(np.float32)
    assert (v32[ci == rows] == 1.0).all()
    x = W.uniform_mt(n, -1, 1, 6).astype(np.float32)
    out = spmv_both(handle, n, rp, ci, v32, x, alpha=-0.5, beta=2.0,
                    y0=W.uniform_mt(n, -1, 1, 7).astype(np.float32))
    assert out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


def test_slots_refused_where_it_does_not_apply(handle):
    import torch
    from monolish_b200.device import Crs
    n, rp, ci, v = W.zipf(5000, seed=2, maxlen=50)  # rows longer than 8 entries
    v = v.astype(np.float32)
    x = W.uniform_mt(n, -1, 1, 8).astype(np.float32)
    out = spmv_both(handle, n, rp, ci, v, x)
    assert out[0][0] and not out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    # an unsorted row
    n, rp, ci, v = W.poisson2d(16)
    ci = ci.copy()
    ci[rp[40]], ci[rp[40] + 1] = ci[rp[40] + 1], ci[rp[40]]
    A = Crs(handle, n, n, rp, ci, v.astype(np.float32))
    assert not A.set_layout(1)
    A.close()
    # FP64 plans keep the CRS arrays
    n, rp, ci, v = W.poisson2d(16)
    A = Crs(handle, n, n, rp, ci, v)
    from monolish_b200 import _abi
    with pytest.raises(_abi.MlshError):
        A.set_layout(1)
    A.close()
    del torch
