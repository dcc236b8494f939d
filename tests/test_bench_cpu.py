"""bench.py's reference arm on the CPU: the JSON line carries the contract's
keys (metric, value, unit, impl, cpu_baseline, e2e) on small workloads."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_ref(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3", *args],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("args", [["--workload", "spmv_poisson3d_f64", "--size", "24"],
                                  ["--workload", "precond_sor_cg", "--size", "32"],
                                  ["--workload", "precond_ilu_bicgstab", "--size", "12"]])
def test_reference_arm_json(reference, args):
    out = run_ref(*args)
    assert out["impl"] == "reference"
    for k in ("metric", "value", "unit", "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in out, k
    assert out["value"] > 0 and out["e2e"]["value"] == out["value"]
    assert out["cpu_baseline"]["kind"] in ("reference", "port")
    if "precond_ilu" in args[1]:
        # the reference has no CPU ILU: the oracle's restatement stands in
        assert out["cpu_baseline"]["kind"] == "port" and out["cpu_baseline"]["cores"] == 1


@pytest.mark.parametrize("workload", ["spmv_poisson3d_f64", "cg_poisson2d"])
def test_reference_arm_maps_no_product_library(reference, workload):
    """The reference arm runs only the reference build and the oracle-side
    generator: no library under monolish_b200/lib is mapped."""
    code = (
        "import sys, types, bench\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--workload', '{workload}', "
        "'--size', '16', '--steps', '1', '--warmup', '3']\n"
        "bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "libs = sorted({l.split()[-1] for l in maps.splitlines() if l.endswith('.so')})\n"
        "print('MAPS', [p for p in libs if '/monolish_b200/' in p or '/oracle/' in p])\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("MAPS")][-1]
    assert "monolish_b200/lib" not in line, line
    assert "libmlsh_gen_oracle.so" in line and "libmonolish_cpu.so" in line, line
