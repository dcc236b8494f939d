"""Builds the reference's own test programs for the CRS solve path against
this library's C++ layer (test infrastructure; needs the reference source
tree, named by MONOLISH_REF or the first argument).

The reference's test headers are used unchanged, read in place: a staging
tree under _build/ holds symlinks to them at the relative places their
#include lines expect, next to this directory's test_utils.hpp (the subset
of the reference's helpers they use) and the C++ layer's headers.  Outputs,
all in _build/ (git-ignored): ref_equation, ref_blas and a copy of the
reference's test matrix test.mtx, so the programs run where the reference
tree is absent.

    MONOLISH_REF=<monolish source tree> python tests/cpp/reference_tests/build_reference_tests.py
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "_build")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

EQUATION = ["test/equation/iterative/equation_kernel.hpp"]
BLAS = [f"test/vector/blas/{f}.hpp" for f in ("copy", "axpy", "xpay", "axpyz", "dot", "nrm2")]


def link(src, dst):
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    if os.path.lexists(dst):
        os.remove(dst)
    os.symlink(src, dst)


def build(ref):
    tree = os.path.join(OUT, "tree")
    if os.path.isdir(tree):
        shutil.rmtree(tree)
    for rel in EQUATION + BLAS:
        link(os.path.join(ref, rel), os.path.join(tree, rel))
    link(os.path.join(HERE, "test_utils.hpp"), os.path.join(tree, "test", "test_utils.hpp"))
    # equation_kernel.hpp includes "../include/monolish_*.hpp"
    link(os.path.join(ROOT, "monolish_b200", "cpp", "include"),
         os.path.join(tree, "test", "equation", "include"))
    shutil.copyfile(os.path.join(ref, "test", "test.mtx"), os.path.join(OUT, "test.mtx"))
    lib = os.path.join(ROOT, "monolish_b200", "lib")
    common = ["-std=c++17", "-O2", "-w", "-I", os.path.join(ROOT, "monolish_b200", "cpp", "include"),
              "-I", os.path.join(ROOT, "include"), "-L", lib, "-lmonolish_b200", "-lmlsh",
              "-Wl,-rpath,$ORIGIN/../../../../monolish_b200/lib"]
    for name, sub, main in (("ref_equation", "test/equation/iterative", "equation_main.cpp"),
                            ("ref_blas", "test/vector/blas", "blas_main.cpp")):
        cmd = [CXX, "-I", os.path.join(tree, sub), os.path.join(HERE, main), "-o",
               os.path.join(OUT, name)] + common
        print("+", " ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MONOLISH_REF", "")
    if not ref or not os.path.isdir(os.path.join(ref, "test")):
        raise SystemExit("set MONOLISH_REF (or pass the path) to the monolish source tree")
    build(ref)
