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
