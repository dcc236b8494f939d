"""Vector BLAS / VML on the GPU against the reference's golden values and
numpy.  Dots and norms: |err| <= 1e-14 * sum|x_i y_i| (summation order
differs from the reference's CBLAS); elementwise ops: within 1 ulp (the
GPU contracts a*x+y into one FMA)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_golden_blas1(handle):
    g = np.load(os.path.join(GOLDEN, "blas1.npz"))
    x, y = g["x"], g["y"]
    assert abs(handle.dot(dev(x), dev(y)) - float(g["dot"])) <= 1e-14 * np.abs(x * y).sum()
    assert abs(handle.nrm2(dev(x)) - float(g["nrm2"])) <= 1e-14 * float(g["nrm2"])
    for op in ("axpy", "xpay"):
        dy = dev(y)
        getattr(handle, op)(0.75, dev(x), dy)
        np.testing.assert_allclose(dy.cpu().numpy(), g[op], rtol=2.3e-16, atol=1e-16)
    dz = dev(np.zeros_like(x))
    handle.axpyz(0.75, dev(x), dev(y), dz)
    np.testing.assert_allclose(dz.cpu().numpy(), g["axpyz"], rtol=2.3e-16, atol=1e-16)


@pytest.mark.parametrize("n", [0, 1, 7, 1000, 1 << 20, (1 << 22) + 3])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_ops_sizes(handle, n, dt):
    rng = np.random.default_rng(n)
    a = rng.uniform(-1, 1, n).astype(dt)
    b = rng.uniform(0.5, 2, n).astype(dt)
    eps = np.finfo(dt).eps
    d = handle.dot(dev(a), dev(b))
    ref = np.dot(a.astype(np.float64), b.astype(np.float64))
    assert abs(d - ref) <= 1e-14 * max(np.abs(a.astype(np.float64) * b).sum(), 1e-300)
    assert abs(handle.nrm2(dev(a)) - np.linalg.norm(a.astype(np.float64))) <= 1e-14 * max(
        np.linalg.norm(a.astype(np.float64)), 1e-300)
    y = dev(np.zeros(n, dt))
    handle.vsub(dev(a), dev(b), y)
    assert np.array_equal(y.cpu().numpy(), a - b)
    handle.vmul(dev(a), dev(b), y)
    assert np.array_equal(y.cpu().numpy(), a * b)
    handle.vreciprocal(dev(b), y)
    assert np.array_equal(y.cpu().numpy(), (1 / b).astype(dt))
    handle.copy(dev(a), y)
    assert np.array_equal(y.cpu().numpy(), a)
    yy = dev(b.copy())
    handle.axpy(-1.5, dev(a), yy)
    np.testing.assert_allclose(yy.cpu().numpy(), (-1.5 * a.astype(np.float64) + b), rtol=2 * eps,
                               atol=2 * eps)


def test_dot_repeatable_bitwise(handle):
    rng = np.random.default_rng(1)
    a = dev(rng.uniform(-1, 1, 3_000_001))
    b = dev(rng.uniform(-1, 1, 3_000_001))
    vals = {handle.dot(a, b) for _ in range(5)}
    assert len(vals) == 1
