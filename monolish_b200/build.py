"""Build steps for the native libraries (run in-tree; outputs in lib/).

* ``lib/libmlsh.so``      -- the CUDA library behind include/mlsh.h, compiled
  for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
* ``lib/libmlsh_gen.so``  -- the seeded workload generators (host C++).
* ``lib/libmonolish_b200.so`` -- the C++ drop-in layer (monolish's class and
  function names) over the C ABI.
* the checker libraries under ``oracle/`` (``make -C oracle``): the C
  restatement and the generators' oracle-side copy always, the reference CPU
  build when the reference source tree is found (``reference_tree()``).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
CSRC = os.path.join(PKG, "csrc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _run(cmd, cwd=None):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, cwd=cwd, check=True)


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build_cuda(force=False):
    os.makedirs(LIB, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = srcs + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(ROOT, "include", "mlsh.h")]
    out = os.path.join(LIB, "libmlsh.so")
    if not force and _newer(out, deps):
        return out
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-shared", "-o", out, *srcs]
    _run(cmd)
    return out


def build_gen(force=False):
    os.makedirs(LIB, exist_ok=True)
    src = os.path.join(PKG, "gen", "mlsh_gen.cpp")
    out = os.path.join(LIB, "libmlsh_gen.so")
    if not force and _newer(out, [src]):
        return out
    _run([CXX, "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", out, src])
    return out


def build_facade(force=False):
    """C++ drop-in layer: monolish's API over the C ABI."""
    cpp = os.path.join(PKG, "cpp")
    srcs = sorted(glob.glob(os.path.join(cpp, "src", "*.cpp")))
    if not srcs:
        return None
    hdrs = sorted(glob.glob(os.path.join(cpp, "include", "**", "*.hpp"), recursive=True))
    out = os.path.join(LIB, "libmonolish_b200.so")
    if not force and _newer(out, srcs + hdrs + [os.path.join(LIB, "libmlsh.so")]):
        return out
    _run([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-I", os.path.join(cpp, "include"),
          "-I", os.path.join(ROOT, "include"), "-o", out, *srcs, "-L", LIB, "-lmlsh",
          "-Wl,-rpath,$ORIGIN"])
    return out


def reference_tree():
    """The monolish source tree the checker libraries are built from:
    ``MONOLISH_REF`` when set, else a checkout named ``reference`` beside
    this repository; "" when neither holds a ``src/`` directory."""
    for ref in (os.environ.get("MONOLISH_REF", ""),
                os.path.join(os.path.dirname(ROOT), "reference")):
        if ref and os.path.isdir(os.path.join(ref, "src")):
            return ref
    return ""


def build_oracle():
    """Checker libraries (test infrastructure only).

    The C restatement and the oracle-side copy of the generators always; the
    reference CPU build only when a monolish source tree is found (its
    ``src/`` is compiled in place, outputs go to ``oracle/_ref``)."""
    oracle = os.path.join(ROOT, "oracle")
    target = ["restatement", "gen"]
    ref = reference_tree()
    extra = []
    if ref:
        target.append("ref")
        extra.append(f"REF={ref}")
    elif not os.path.exists(os.path.join(oracle, "_ref", "libmlsh_refcapi.so")):
        print("oracle/_ref not built: set MONOLISH_REF to a monolish source tree", flush=True)
    _run(["make", "-s", "-j", str(os.cpu_count() or 4), *target, *extra], cwd=oracle)


def build_reference_tests():
    """The reference's own test programs against the C++ layer (test
    infrastructure), when the reference source tree is found."""
    ref = reference_tree()
    if not ref or not os.path.isdir(os.path.join(ref, "test")):
        return
    script = os.path.join(ROOT, "tests", "cpp", "reference_tests", "build_reference_tests.py")
    _run([sys.executable, script, ref])


def build_all(force=False):
    build_cuda(force)
    build_gen(force)
    build_facade(force)
    build_oracle()
    build_reference_tests()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
