"""mlsh_dot_noalloc -- the dot product for callers that cannot allocate
device memory (a framework that owns the device memory through its own pool,
a latency-critical loop that cannot take cudaMalloc's implicit
synchronisation).  Its scratch is a static device array shared by every
call, so this test makes two calls in a row (different sizes, so the second
reuses what the first left in the array) and checks each against the
allocating entry point mlsh_dot_device, through the C ABI.  Both run the
same grid and summation order on the same stream, so their results must be
identical bit for bit; against numpy's FP64 dot the bar is the one the other
dot tests use, |err| <= 1e-14 * sum|x_i y_i|.

Named test_zz_* so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from monolish_b200 import _abi

pytestmark = pytest.mark.gpu


def _dot_pair(handle, lib, x, y, dtype_code):
    import torch
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = x.numel()
    _abi.check(lib.mlsh_dot_noalloc(dtype_code, n, x.data_ptr(), y.data_ptr(),
                                    out.data_ptr(), stream), "mlsh_dot_noalloc")
    _abi.check(lib.mlsh_dot_device(handle.h, dtype_code, n, x.data_ptr(), y.data_ptr(),
                                   out.data_ptr() + 8), "mlsh_dot_device")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_dot_noalloc_matches_dot_device_twice(handle):
    import torch
    lib = _abi.load()
    rng = np.random.default_rng(42)
    cases = [
        (np.float64, _abi.F64, 3_000_001),  # many CTAs: fills most of the scratch
        (np.float32, _abi.F32, 1_000),      # one CTA: reuses what the first call left
    ]
    for dt, code, n in cases:
        a = rng.uniform(-1, 1, n).astype(dt)
        b = rng.uniform(-1, 1, n).astype(dt)
        x = torch.from_numpy(a).cuda()
        y = torch.from_numpy(b).cuda()
        got, ref = _dot_pair(handle, lib, x, y, code)
        tol = 1e-14 * np.abs(a.astype(np.float64) * b.astype(np.float64)).sum()
        assert np.isfinite(got)
        assert got == ref, (dt, n, got, ref)
        exact = float(np.dot(a.astype(np.float64), b.astype(np.float64)))
        assert abs(got - exact) <= tol


def test_dot_noalloc_empty_is_zero():
    import torch
    lib = _abi.load()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _abi.check(lib.mlsh_dot_noalloc(_abi.F64, 0, None, None, out.data_ptr(), stream),
               "mlsh_dot_noalloc")
    torch.cuda.synchronize()
    assert out.item() == 0.0


def test_dot_noalloc_rejects_bad_arguments():
    import torch
    lib = _abi.load()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.mlsh_dot_noalloc(_abi.F64, -1, None, None, out.data_ptr(), None) == \
        _abi.ERR_INVALID_ARG
    assert lib.mlsh_dot_noalloc(7, 10, out.data_ptr(), out.data_ptr(), out.data_ptr(),
                                None) == _abi.ERR_INVALID_ARG
