"""B200-native (sm_100a) sparse iterative-solve path with monolish's API.

The product is the CUDA library ``lib/libmlsh.so`` behind the C ABI in
``include/mlsh.h`` and the C++ drop-in layer ``lib/libmonolish_b200.so``
(monolish's ``matrix::CRS``, ``vector``, ``blas::matvec/dot/nrm2/...`` and
``equation::CG/BiCGSTAB`` names).  This Python package holds the build
script, the generators' bindings and a thin ctypes harness used by the
tests and the benchmark.
"""
from . import _abi  # noqa: F401

__all__ = ["_abi"]
