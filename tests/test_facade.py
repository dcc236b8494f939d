"""The C++ drop-in layer: programs written against monolish's API
(tests/cpp/*.cpp) compile against monolish_b200/cpp/include and link
libmonolish_b200.so; on a GPU they run and pass their own checks."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "monolish_b200", "lib")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def compile_prog(name, outdir):
    src = os.path.join(ROOT, "tests", "cpp", f"{name}.cpp")
    exe = os.path.join(outdir, name)
    cmd = [CXX, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "monolish_b200", "cpp", "include"),
           "-I", os.path.join(ROOT, "include"), src, "-o", exe, "-L", LIB, "-lmonolish_b200",
           "-lmlsh", f"-Wl,-rpath,{LIB}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def write_mm(path, n, rp, ci, v):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {len(v)}\n")
        for i in range(n):
            for j in range(rp[i], rp[i + 1]):
                f.write(f"{i + 1} {int(ci[j]) + 1} {float(v[j])!r}\n")


@pytest.fixture(scope="module")
def progs(tmp_path_factory):
    if not os.path.exists(os.path.join(LIB, "libmonolish_b200.so")):
        from monolish_b200 import build
        build.build_facade()
    d = tmp_path_factory.mktemp("cpp")
    return {n: compile_prog(n, str(d)) for n in ("equation_test", "blas_test", "view_test")}, d


def test_dropin_programs_compile(progs):
    exes, _ = progs
    assert all(os.path.exists(e) for e in exes.values())


@pytest.mark.gpu
def test_dropin_blas(progs, cuda):
    exes, _ = progs
    r = subprocess.run([exes["blas_test"]], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_equation(progs, cuda):
    from monolish_b200 import workloads as W
    exes, d = progs
    tri = os.path.join(d, "tridiag.mtx")
    write_mm(tri, 3, np.array([0, 2, 5, 7]), np.array([0, 1, 0, 1, 2, 1, 2]),
             np.array([2.0, -1, -1, 2, -1, -1, 2]))
    n, rp, ci, v = W.vardiff2d(24, 19, 3, 1)
    big = os.path.join(d, "vardiff.mtx")
    write_mm(big, n, rp, ci, v)
    for f in (tri, big):
        r = subprocess.run([exes["equation_test"], f], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_view1d(progs, cuda):
    exes, _ = progs
    r = subprocess.run([exes["view_test"]], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


REF_TESTS = os.path.join(ROOT, "tests", "cpp", "reference_tests", "_build")


@pytest.mark.gpu
@pytest.mark.parametrize("prog,args", [("ref_equation", ["test.mtx", "1"]),
                                       ("ref_blas", ["100"]), ("ref_blas", ["123456"])])
def test_reference_test_programs(cuda, prog, args):
    """The reference's own test programs for this path -- the solver test
    (test/equation/iterative/equation_kernel.hpp: CG and BiCGSTAB, none and
    Jacobi, CRS<double> and CRS<float>, on the reference's test.mtx, answer
    checked against ones) and the device forms of its vector BLAS tests
    (test/vector/blas) -- compiled unchanged against this library's C++
    layer by tests/cpp/reference_tests/build_reference_tests.py."""
    exe = os.path.join(REF_TESTS, prog)
    if not os.path.exists(exe):
        pytest.skip("reference test programs not built (needs the reference tree)")
    argv = [exe] + [os.path.join(REF_TESTS, a) if a.endswith(".mtx") else a for a in args]
    r = subprocess.run(argv, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout[-3000:] + r.stderr[-2000:]
