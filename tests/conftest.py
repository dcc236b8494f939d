"""Test configuration.

Markers:
  gpu -- needs a CUDA device (run with ``-m gpu`` on a B200); everything else
         runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    from monolish_b200 import build
    lib = os.path.join(ROOT, "monolish_b200", "lib")
    if not os.path.exists(os.path.join(lib, "libmlsh_gen.so")):
        build.build_gen()
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "libmlsh_oracle.so")):
        import subprocess
        subprocess.run(["make", "-s", "restatement"], cwd=os.path.join(ROOT, "oracle"),
                       check=True)


_ensure_built()


@pytest.fixture(scope="session")
def restatement():
    import oracle
    return oracle.restatement()


@pytest.fixture(scope="session")
def reference():
    import oracle
    ref = oracle.reference_or_none()
    if ref is None:
        pytest.skip("reference CPU build (oracle/_ref) not present")
    return ref


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda")


@pytest.fixture(scope="session")
def handle(cuda):
    from monolish_b200.device import Handle
    h = Handle()
    yield h
    h.close()
