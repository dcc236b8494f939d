"""The C ABI library loads and exports every symbol include/mlsh.h
declares; host-side behaviour that needs no GPU.  CPU only."""
import ctypes
import os
import re

import pytest

from monolish_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(mlsh_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_abi.LIB_PATH):
        pytest.skip("libmlsh.so not built")
    lib = ctypes.CDLL(_abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    names = set(declared_symbols())
    assert names <= set(_abi.SIGNATURES), sorted(names - set(_abi.SIGNATURES))


def test_status_strings_and_defaults():
    if not os.path.exists(_abi.LIB_PATH):
        pytest.skip("libmlsh.so not built")
    lib = _abi.load()
    assert lib.mlsh_version() >= 100
    for code in (0, -1, -2, -3, -4, -10, -20, -21, -22, -23, -24, -25):
        assert lib.mlsh_status_string(code)
    o = _abi.SolverOpts()
    assert lib.mlsh_solver_opts_default(ctypes.byref(o)) == 0
    assert o.tol == 1e-8 and o.miniter == 0 and o.precond == 1
    # invalid arguments are rejected before any device work
    assert lib.mlsh_destroy(None) == _abi.ERR_INVALID_ARG
    assert lib.mlsh_spmv(None, None, 1.0, None, 0.0, None) == _abi.ERR_INVALID_ARG
    assert lib.mlsh_cg_solve(None, None, None, None, None, None) == _abi.ERR_INVALID_ARG


def test_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = _abi.load()
    h = ctypes.c_void_p()
    assert lib.mlsh_create(ctypes.byref(h)) == _abi.ERR_NO_DEVICE
