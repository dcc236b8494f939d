#!/usr/bin/env python
"""Benchmark of the sparse solve path on B200 (one JSON line on rank 0).

Default workload: CRS SpMV y = A*x in FP64 on the 3D 7-point Laplacian
256^3 (n = 16,777,216, nnz = 117,047,296; 1.74 GB of algorithmic traffic
per SpMV, larger than the 126 MB L2, so no flush is needed between steps).
A "step" is one SpMV over the whole matrix.  The metric is achieved HBM
GB/s with algorithmic bytes  nnz*(V+4) + (n+1)*4 + 2*n*X  per SpMV.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

* ``value``  -- GB/s of the device-resident SpMV (inputs already in HBM),
  CUDA events on the launching stream, max over ranks; N GPUs run
  independent replicas (the single-system SpMV does not shard without a
  halo exchange), so the whole-job value is the sum over ranks.
* ``e2e``    -- the same metric through the C ABI with host buffers: every
  step copies x host->device from pinned memory, runs the SpMV and reads y
  back (the matrix stays resident, as after the reference's ``send()``).
* ``roofline`` -- the SpMV kernel's algorithmic bytes per launch / average
  launch time against the measured HBM copy bandwidth; ``traffic`` is DRAM
  bytes per launch from the committed ncu summary of this workload.
* ``cpu_baseline`` -- the reference's own CPU SpMV (OpenMP row loop,
  compiled from the reference sources) on the same matrix and the box's
  host cores.
* ``--impl reference`` -- times that reference CPU SpMV as the run's arm.

Other workloads (``--workload``): spmv_poisson3d_f32, spmv_zipf_f64,
spmv_zipf_f32, cg_poisson2d (128x128 Jacobi-CG to 1e-10, solves/s),
bicgstab_convdiff (160^3 Jacobi-BiCGSTAB to 1e-10, solves/s).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC_SPMV = "SpMV HBM GB/s"
NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e, nominal
METRIC_SOLVE = "solves/s at 1e-10 rel. residual"

WORKLOADS = {
    "spmv_poisson3d_f64": dict(kind="spmv", matrix="poisson3d", m=256, dtype="f64"),
    "spmv_poisson3d_f32": dict(kind="spmv", matrix="poisson3d", m=256, dtype="f32"),
    "spmv_zipf_f64": dict(kind="spmv", matrix="zipf", n=4194304, dtype="f64"),
    "spmv_zipf_f32": dict(kind="spmv", matrix="zipf", n=4194304, dtype="f32"),
    "cg_poisson2d": dict(kind="cg", matrix="poisson2d", m=128, dtype="f64"),
    "bicgstab_convdiff": dict(kind="bicgstab", matrix="convdiff3d", m=160, dtype="f64"),
    "batch_cg": dict(kind="batch", matrix="diffusion_batch", count=2048, dtype="f64"),
    "serve_stream": dict(kind="serve", matrix="serve", count=200, budget=8 << 30,
                         dtype="f64"),
    # CG / BiCGSTAB with the triangular-sweep preconditioners (SOR, IC(0), ILU(0))
    "precond_sor_cg": dict(kind="precond", solver="cg", pc="sor", matrix="poisson2d", m=128,
                           dtype="f64"),
    "precond_ic_cg": dict(kind="precond", solver="cg", pc="ic", matrix="poisson3d", m=128,
                          dtype="f64"),
    "precond_ilu_bicgstab": dict(kind="precond", solver="bicgstab", pc="ilu",
                                 matrix="convdiff3d", m=96, dtype="f64"),
}
METRIC_PRECOND = "preconditioned solves/s at 1e-10 rel. residual"
PC_KIND = {"sor": 2, "ic": 3, "ilu": 4}
METRIC_BATCH = "solves/s at 1e-8 rel. residual, 2,048-system batch"


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def describe(wl):
    if wl.get("size"):
        wl = dict(wl, **({"n": wl["size"]} if wl["matrix"] == "zipf" else {"m": wl["size"]}))
    if wl["kind"] == "precond":
        mat = {"poisson2d": f"2D 5-point Poisson {wl['m']}x{wl['m']} (x_true U[-1,1] seed 0)",
               "poisson3d": f"3D 7-point Laplacian {wl['m']}^3 (x_true U[-1,1] seed 1)",
               "convdiff3d": f"3D upwind convection-diffusion {wl['m']}^3, cell Peclet 10 "
                             "(x_true U[-1,1] seed 2)"}[wl["matrix"]]
        pcn = {"sor": "SOR (omega 1.9)", "ic": "IC(0)", "ilu": "ILU(0)"}[wl["pc"]]
        return (f"{wl['solver'].upper() if wl['solver'] == 'cg' else 'BiCGSTAB'} "
                f"preconditioned by {pcn} on {mat}, tol 1e-10*||b||, FP64")
    if wl["matrix"] == "poisson3d":
        return f"3D 7-point Laplacian {wl['m']}^3 CRS<{'double' if wl['dtype'] == 'f64' else 'float'}>"
    if wl["matrix"] == "zipf":
        return (f"Zipf(2) rows n={wl['n']}, lengths 1..10000, uniform sorted columns, "
                f"U[-1,1] values (seed 1), CRS<{'double' if wl['dtype'] == 'f64' else 'float'}>")
    if wl["matrix"] == "poisson2d":
        return f"2D 5-point Poisson {wl['m']}x{wl['m']}, Jacobi-CG, x_true U[-1,1] seed 0, tol 1e-10*||b||"
    if wl["matrix"] == "convdiff3d":
        return (f"3D upwind convection-diffusion {wl['m']}^3, cell Peclet 10, Jacobi-BiCGSTAB, "
                f"x_true U[-1,1] seed 2, tol 1e-10*||b||")
    return wl["matrix"]


def make_matrix(wl):
    from monolish_b200 import workloads as W
    if wl.get("size"):
        wl = dict(wl, **({"n": wl["size"]} if wl["matrix"] == "zipf" else {"m": wl["size"]}))
    if wl["matrix"] == "poisson3d":
        n, rp, ci, v = W.poisson3d(wl["m"])
        x = W.uniform_fast(n, -1.0, 1.0, 1)
    elif wl["matrix"] == "zipf":
        n, rp, ci, v = W.zipf(wl["n"], seed=1)
        x = W.uniform_fast(n, -1.0, 1.0, 1)
    elif wl["matrix"] == "poisson2d":
        n, rp, ci, v = W.poisson2d(wl["m"])
        x = W.uniform_mt(n, -1.0, 1.0, 0)
    elif wl["matrix"] == "convdiff3d":
        n, rp, ci, v = W.convdiff3d(wl["m"], peclet=10.0)
        x = W.uniform_mt(n, -1.0, 1.0, 2)
    else:
        raise ValueError(wl)
    if wl["dtype"] == "f32":
        v = v.astype(np.float32)
        x = x.astype(np.float32)
    return n, rp, ci, v, x


def spmv_bytes(n, nnz, vsz):
    return nnz * (vsz + 4) + (n + 1) * 4 + 2 * n * vsz


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.path = None
        self.gpu = gpu_index
        self.t0 = self.t1 = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def mark(self, which):
        setattr(self, which, time.time())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [s.strip() for s in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for nm, val in zip(names[1:], f[5:9]):
                    if val.lower() == "active":
                        reasons.add(nm)
            os.unlink(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(workload):
    """DRAM bytes per launch of the SpMV kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{workload}.traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


# ------------------------------------------------------ host-side inputs
def host_matvec(rp, ci, v, x):
    """y = A x on the host in FP64 (scipy CSR): builds right-hand sides and
    checks true residuals; never on a timed path."""
    import scipy.sparse as sp
    n = len(rp) - 1
    A = sp.csr_matrix((np.asarray(v, np.float64), ci, rp), shape=(n, len(x)))
    return A @ np.asarray(x, np.float64)


def true_relres(rp, ci, v, b, x):
    r = b - host_matvec(rp, ci, v, x)
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(r)) / (nb if nb > 0 else 1.0)


# ------------------------------------------------------------- CPU leg
def cpu_reference_spmv(rp, ci, v, x, reps, threads):
    """The reference's CPU SpMV (oracle/_ref build, OpenMP row loop)."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    import oracle
    ref = oracle.reference_or_none()
    if ref is not None:
        ref.set_threads(threads)
        _, mean_s, best_s = ref.spmv(rp, ci, v, x, reps=reps)
        return mean_s, "reference", threads
    port = oracle.restatement()
    t0 = time.perf_counter()
    for _ in range(reps):
        port.spmv(rp, ci, v, x)
    return (time.perf_counter() - t0) / reps, "port", 1


# ------------------------------------------------------------- our arm
def run_spmv(args, wl, rank, world, local):
    import torch
    import torch.distributed as dist
    from monolish_b200 import _abi
    from monolish_b200 import device as D

    torch.cuda.set_device(local)
    n, rp, ci, v, x = make_matrix(wl)
    nnz = int(rp[-1])
    vsz = 8 if wl["dtype"] == "f64" else 4
    B = spmv_bytes(n, nnz, vsz)
    h = D.Handle()
    A = D.Crs(h, n, n, rp, ci, v, validate=False)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty(n, dtype=dx.dtype, device="cuda")
    # consecutive timed launches read two different copies of x, so no
    # launch finds the x of the one before it in L2
    dx2 = dx.clone()
    stream = torch.cuda.current_stream()
    lib, hh, plan = h.lib, h.h, A.plan
    xps, yp = (dx.data_ptr(), dx2.data_ptr()), dy.data_ptr()
    nlaunch = [0]

    def launch():
        st = lib.mlsh_spmv(hh, plan, 1.0, xps[nlaunch[0] & 1], 0.0, yp)
        nlaunch[0] += 1
        if st != 0:
            raise _abi.MlshError(st, "spmv")

    # setup (untimed): pick the SpMV kernel variant for this matrix
    if args.variant >= 0:
        A.set_variant(args.variant)
        variant = args.variant
    else:
        variant, _ = A.autotune(dx, dy)
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    if not args.quick:
        clocks.start()
        # keep the sampler running over a warm-up soak so short timed regions
        # still have clock samples of the same work around them
        soak_end = time.time() + 1.0
        while time.time() < soak_end:
            launch()
            torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        launch()
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    cl = clocks.stop()
    h.sync()

    # ---- end to end through the C ABI with host buffers: every step copies
    # its x in from pinned memory, runs the SpMV and copies its y out, the
    # copies through the library's own stream-ordered mlsh_memcpy_*_async on
    # handles bound to a copy-in and a copy-out stream.  Two device buffer
    # pairs let step k+1's copy-in run while step k computes and copies out
    # (PCIe is full duplex).
    del dx2
    hx = torch.from_numpy(x).pin_memory()
    hys = [torch.empty(n, dtype=dx.dtype).pin_memory() for _ in range(2)]
    hy = hys[0]
    xs = [dx, torch.empty_like(dx)]
    ys = [dy, torch.empty_like(dy)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    h_in, h_out = D.Handle(stream=s_in.cuda_stream), D.Handle(stream=s_out.cuda_stream)
    xbytes = n * dx.element_size()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_sp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    e2e_steps = 0 if args.quick else max(1, min(args.steps, 50))
    e2e_ms = 1.0

    def e2e_step(k):
        j = k % 2
        if k >= 2:
            s_in.wait_event(ev_sp[j])          # x_j no longer read by step k-2
        _abi.check(lib.mlsh_memcpy_h2d_async(h_in.h, xs[j].data_ptr(), hx.data_ptr(),
                                             xbytes), "memcpy_h2d_async")
        ev_in[j].record(s_in)
        stream.wait_event(ev_in[j])
        if k >= 2:
            stream.wait_event(ev_out[j])       # y_j copied out by step k-2
        st = lib.mlsh_spmv(hh, plan, 1.0, xs[j].data_ptr(), 0.0, ys[j].data_ptr())
        if st != 0:
            raise _abi.MlshError(st, "spmv")
        ev_sp[j].record(stream)
        s_out.wait_event(ev_sp[j])
        _abi.check(lib.mlsh_memcpy_d2h_async(h_out.h, hys[j].data_ptr(), ys[j].data_ptr(),
                                             xbytes), "memcpy_d2h_async")
        ev_out[j].record(s_out)
        return j

    if e2e_steps:
        for k in range(2):
            e2e_step(k)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        last = 0
        for k in range(e2e_steps):
            last = e2e_step(k)
        stream.wait_event(ev_out[last])
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        hy = hys[last]
        if world > 1:
            dist.barrier()
    else:
        hy.copy_(dy)
    h_in.close()
    h_out.close()

    # correctness spot check: FP64 numpy row dots on a sample of rows
    y = hy.numpy()
    rows = np.linspace(0, n - 1, 2048).astype(np.int64)
    ref_rows = np.array([np.dot(v[rp[i]:rp[i + 1]].astype(np.float64),
                                x[ci[rp[i]:rp[i + 1]]].astype(np.float64)) for i in rows])
    tol = 1e-12 if vsz == 8 else 1e-4
    scale = np.array([np.abs(v[rp[i]:rp[i + 1]] * x[ci[rp[i]:rp[i + 1]]]).sum() for i in rows])
    ok = bool(np.all(np.abs(y[rows] - ref_rows) <= tol * np.maximum(scale, 1e-30)))

    if world > 1:
        t = torch.tensor([ms, e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])
    per_launch_s = ms / 1e3 / args.steps
    value = world * B * args.steps / (ms / 1e3) / 1e9
    e2e_value = world * B * e2e_steps / (e2e_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    achieved = B / per_launch_s / 1e9
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            reps = 5
            threads = os.cpu_count() or 1
            sec, kind, cores = cpu_reference_spmv(rp, ci, v, x, reps, threads)
            cpu = {"value": round(B / sec / 1e9, 3), "unit": "GB/s", "cores": cores,
                   "kind": kind,
                   "sample": f"{reps} full SpMVs of the same matrix (mean), {cores} threads"}
        info = A.info()
        out = {
            "metric": METRIC_SPMV, "value": round(value, 2), "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
            "data": "synthetic (seeded generators)",
            "config": {"workload": describe(wl), "n": n, "nnz": nnz,
                       "bytes_per_step": B, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (the matrix streamed L2 "
                             "evict-first); consecutive launches read two different "
                             "copies of x, so none finds the previous launch's x in L2",
                       "n_tiles": info["n_tiles"], "n_long_rows": info["n_long_rows"],
                       "spmv_variant": variant, "short_row_limit": A.tuning()[1]},
            "e2e": {"value": round(e2e_value, 2), "unit": "GB/s",
                    "h2d_bytes_per_step": n * vsz, "d2h_bytes_per_step": n * vsz,
                    "steps": e2e_steps,
                    "note": "x in from pinned host memory and y out every step through "
                            "mlsh_memcpy_h2d_async / mlsh_memcpy_d2h_async; step k+1's "
                            "copy-in overlaps step k's SpMV and copy-out (two buffer pairs)"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_kind": peak_kind,
                         "traffic": profile_traffic(args.workload)},
            "gpu_launches": args.steps,
            "check": {"rows_checked": len(rows), "ok": ok},
        }
        if cpu:
            out["cpu_baseline"] = cpu
        if cl:
            out["clocks"] = cl
    A.close()
    h.close()
    return out


def run_solve(args, wl, rank, world, local):
    import torch
    import torch.distributed as dist
    from monolish_b200 import device as D

    torch.cuda.set_device(local)
    n, rp, ci, v, xt = make_matrix(wl)
    b = host_matvec(rp, ci, v, xt)
    tol = 1e-10 * float(np.linalg.norm(b))
    h = D.Handle()
    A = D.Crs(h, n, n, rp, ci, v, validate=False)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    base_fn = D.cg_solve if wl["kind"] == "cg" else D.bicgstab_solve
    inner_tol = 1e-4 if args.inner_tol is None else args.inner_tol
    mixed_fn = D.cg_solve_mixed if wl["kind"] == "cg" else D.bicgstab_solve_mixed
    engine = {"auto": 0, "kernels": 1, "cluster": 2}[args.engine]

    def plain_fn(A_, b_, x_, tol_, maxiter_):
        return base_fn(A_, b_, x_, tol_, maxiter_, engine=engine,
                       cluster_rows=args.cluster_rows, use_graph=not args.eager)

    def fn(A_, b_, x_, tol_, maxiter_):
        if args.precision == "mixed":
            return mixed_fn(A_, b_, x_, tol_, maxiter_, inner_tol=inner_tol, engine=engine,
                            use_graph=not args.eager)
        return plain_fn(A_, b_, x_, tol_, maxiter_)

    stream = torch.cuda.current_stream()
    # the plain FP64 solve, timed beside the mixed one for the speed-up
    plain_ms = None
    if args.precision == "mixed" and not args.quick:
        for _ in range(args.warmup):
            dx.zero_()
            rp_res = plain_fn(A, db, dx, tol, 20000)
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            dx.zero_()
            rp_res = plain_fn(A, db, dx, tol, 20000)
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = p0.elapsed_time(p1) / args.steps
        plain_rel = true_relres(rp, ci, v, b, dx.cpu().numpy())
    for _ in range(args.warmup):
        dx.zero_()
        r = fn(A, db, dx, tol, 20000)
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        dx.zero_()
        r = fn(A, db, dx, tol, 20000)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cl = clocks.stop()
    rel = true_relres(rp, ci, v, b, dx.cpu().numpy())
    # end to end: b from pinned host memory, x back to host, per solve
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(n, dtype=torch.float64).pin_memory()
    e0.record(stream)
    for _ in range(args.steps):
        db.copy_(hb, non_blocking=True)
        dx.zero_()
        r = fn(A, db, dx, tol, 20000)
        hx.copy_(dx, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms, e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])
    out = None
    if rank == 0:
        nnz = int(rp[-1])
        B_it = spmv_bytes(n, nnz, 8) - 2 * n * 8 + 13 * n * 8 if wl["kind"] == "cg" else \
            2 * (spmv_bytes(n, nnz, 8) - 2 * n * 8) + 22 * n * 8
        per_solve_s = ms / 1e3 / args.steps
        total_bytes = B_it * r.iters
        if args.precision == "mixed":
            # inner iterations in FP32 (V = X = 4 bytes), one FP64 residual
            # (SpMV + x update) per outer step
            # the FP32 copy's matrix bytes per SpMV in the layout it uses
            import ctypes
            lay, mb = ctypes.c_int(), ctypes.c_int64()
            h.lib.mlsh_csr_plan_storage(A.plan, 1, ctypes.byref(lay), ctypes.byref(mb))
            B_A32 = int(mb.value) if mb.value > 0 else nnz * 8 + (n + 1) * 4
            B_A64 = nnz * 12 + (n + 1) * 4
            # BiCGSTAB with D^-1 folded into the FP32 values: 19 vector passes
            B_it32 = (B_A32 + 13 * n * 4) if wl["kind"] == "cg" else (2 * B_A32 + 19 * n * 4)
            total_bytes = B_it32 * r.iters + (r.outer + 1) * (B_A64 + 5 * n * 8)
            fp32_layout = {0: "CRS", 1: "offset slots"}.get(lay.value, "none")
        achieved = total_bytes / per_solve_s / 1e9
        peak, peak_kind = measured_peak()
        out = {
            "metric": METRIC_SOLVE, "value": round(world * args.steps / (ms / 1e3), 3),
            "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generators)",
            "config": {"workload": describe(wl), "n": n, "nnz": nnz, "iters": r.iters,
                       "status": r.status, "true_rel_residual": rel,
                       "engine": args.engine, "cluster_rows": args.cluster_rows,
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(world * args.steps / (e2e_ms / 1e3), 3), "unit": "solves/s",
                    "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_kind": peak_kind, "traffic": None,
                         "note": "whole-solve algorithmic bytes (fused minimum) / solve time"},
            "gpu_launches": args.steps * (r.iters * (3 if wl["kind"] == "cg" else 5) + 3),
        }
        if args.precision == "mixed":
            out["dtype"] = "f32 inner / f64 refinement"
            out["config"]["precision"] = "mixed: FP32 inner (tol 1e-4 rel), FP64 outer"
            out["config"]["fp32_layout"] = fp32_layout
            out["config"]["fp32_matrix_bytes_per_spmv"] = B_A32
            out["config"]["outer_steps"] = r.outer
            out["roofline"]["note"] = ("algorithmic bytes: FP32 inner iterations (the FP32 "
                                       "copy's matrix bytes in its layout + 19 vector passes "
                                       "of 4 bytes) plus an FP64 residual per outer step, / "
                                       "solve time")
            out["config"]["inner_tol"] = inner_tol
            if plain_ms is not None:
                out["plain_fp64"] = {"value": round(1e3 / plain_ms, 3), "unit": "solves/s",
                                     "iters": rp_res.iters, "true_rel_residual": plain_rel,
                                     "speedup_of_mixed": round(plain_ms / (ms / args.steps),
                                                               3)}
                # the same mixed solve at other inner tolerances: the FP32
                # iteration's attainable accuracy is about u32 * cond(A D^-1),
                # so inner tolerances near it cost extra FP32 iterations
                sweep = []
                for itol in (() if getattr(args, "no_sweep", False) else (1e-1, 1e-2, 1e-3)):
                    if itol == inner_tol:
                        continue
                    for _ in range(2):
                        dx.zero_()
                        mixed_fn(A, db, dx, tol, 20000, inner_tol=itol, engine=engine)
                    torch.cuda.synchronize()
                    e0.record(stream)
                    for _ in range(args.steps):
                        dx.zero_()
                        rs = mixed_fn(A, db, dx, tol, 20000, inner_tol=itol, engine=engine)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    mt = e0.elapsed_time(e1) / args.steps
                    sweep.append({"inner_tol": itol, "ms_per_solve": round(mt, 3),
                                  "iters": rs.iters, "outer": rs.outer, "status": rs.status,
                                  "true_rel_residual": true_relres(rp, ci, v, b,
                                                                   dx.cpu().numpy()),
                                  "speedup_vs_plain_fp64": round(plain_ms / mt, 3)})
                if sweep:
                    out["inner_tol_sweep"] = sweep
        if world == 1 and not args.no_cpu:
            import oracle
            ref = oracle.reference_or_none()
            if ref is not None:
                ref.set_threads(os.cpu_count() or 1)
                st, it, res, xr, sec = getattr(ref, wl["kind"])(rp, ci, v, b, np.zeros(n), tol,
                                                                20000)
                out["cpu_baseline"] = {"value": round(1.0 / sec, 3), "unit": "solves/s",
                                       "cores": os.cpu_count(), "kind": "reference",
                                       "sample": f"1 full solve ({it} iterations)"}
        if cl:
            out["clocks"] = cl
    A.close()
    h.close()
    return out


# ------------------------------------------------------ preconditioners
def precond_apply_bytes(n, nnz, pc):
    """Algorithmic bytes of one apply z = M^{-1} r (both sweeps): the stored
    entries each sweep reads once (value + column; IC reads L and its
    transpose, SOR / ILU the lower and upper halves of one pattern), per row
    and sweep the row pointer and the two split indices, and the vectors
    (right-hand side in, result out; SOR also its multipliers)."""
    entries = nnz + n if pc == "ic" else nnz
    vec = 4 * n * 8 + (2 * n * 8 if pc == "sor" else 0)
    return entries * 12 + 2 * ((n + 1) * 4 + 2 * n * 4) + vec


def run_precond(args, wl, rank, world, local):
    import torch
    import torch.distributed as dist
    from monolish_b200 import device as D

    torch.cuda.set_device(local)
    n, rp, ci, v, xt = make_matrix(wl)
    b = host_matvec(rp, ci, v, xt)
    tol = 1e-10 * float(np.linalg.norm(b))
    kind = PC_KIND[wl["pc"]]
    h = D.Handle()
    A = D.Crs(h, n, n, rp, ci, v, validate=False)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    solve_fn = D.cg_solve_precond if wl["solver"] == "cg" else D.bicgstab_solve_precond

    def solve(A_, pc_, b_, x_, tol_, maxiter_):
        return solve_fn(A_, pc_, b_, x_, tol_, maxiter_, use_graph=not args.eager)

    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # setup: the factorization (IC / ILU) or multipliers (SOR) and schedules
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pc = D.Precond(A, kind)
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3
    lv_lo, lv_up, nblocks = pc.info()
    forms = pc.sweep_form()
    form_names = {0: "sweep_kernel (flags across the GPU)", 1: "sweep_cta_kernel (one CTA)",
                  2: "sweep_ring_kernel (one CTA, record ring)", -1: "none"}
    # one apply (both sweeps) on its own
    r = torch.from_numpy(b / np.linalg.norm(b)).cuda()
    z = torch.empty_like(r)
    for _ in range(args.warmup):
        pc.apply(r, z)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        pc.apply(r, z)
    e1.record(stream)
    torch.cuda.synchronize()
    apply_ms = e0.elapsed_time(e1) / args.steps
    for _ in range(args.warmup):
        dx.zero_()
        res = solve(A, pc, db, dx, tol, 20000)
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        dx.zero_()
        res = solve(A, pc, db, dx, tol, 20000)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cl = clocks.stop()
    rel = true_relres(rp, ci, v, b, dx.cpu().numpy())
    # end to end as a user of the reference API runs it: b from pinned host
    # memory, the preconditioner built (create_precond, done by every
    # reference solve), the solve, x back to the host
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        db.copy_(hb, non_blocking=True)
        dx.zero_()
        pc2 = D.Precond(A, kind)
        solve(A, pc2, db, dx, tol, 20000)
        hx.copy_(dx, non_blocking=True)
        torch.cuda.synchronize()
        pc2.close()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    if world > 1:
        t = torch.tensor([ms, e2e_ms / e2e_steps * args.steps], device="cuda",
                         dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
    out = None
    if rank == 0:
        nnz = int(rp[-1])
        B_apply = precond_apply_bytes(n, nnz, wl["pc"])
        achieved = B_apply / (apply_ms / 1e3) / 1e9
        peak, peak_kind = measured_peak()
        hops = lv_lo + lv_up
        out = {
            "metric": METRIC_PRECOND, "value": round(world * args.steps / (ms / 1e3), 3),
            "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generators)",
            "config": {"workload": describe(wl), "n": n, "nnz": nnz, "iters": res.iters,
                       "status": res.status, "true_rel_residual": rel,
                       "precond_setup_ms": round(setup_ms, 2),
                       "apply_ms": round(apply_ms, 4),
                       "sweep_levels": [lv_lo, lv_up], "row_blocks": nblocks,
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e_steps / (e2e_ms / 1e3), 3), "unit": "solves/s",
                    "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8,
                    "note": "includes building the preconditioner, as every reference solve "
                            "does"},
            "roofline": {"bound": "latency", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_kind": peak_kind, "traffic": None,
                         "kernel": f"lower: {form_names[forms[0]]}; upper: "
                                   f"{form_names[forms[1]]} (one apply)",
                         "bytes_per_apply": B_apply,
                         "us_per_level": round(apply_ms * 1e3 / max(hops, 1), 2),
                         "note": "algorithmic bytes of one apply / apply time against HBM; the "
                                 "sweeps are bound by their dependency chains: an apply is "
                                 f"{hops} block levels long, each one wait for other warps' "
                                 "results"},
            # per iteration: CG 6 (SpMV, x/r update, 2 sweeps, z.r, p update),
            # BiCGSTAB 9 (p, 2 sweeps, SpMV, s, 2 sweeps, SpMV, x/r); set-up of a
            # solve: CG 4 (SpMV, 2 sweeps, init), BiCGSTAB 2 (SpMV, init)
            "gpu_launches": args.steps * (res.iters * (6 if wl["solver"] == "cg" else 9) +
                                          (4 if wl["solver"] == "cg" else 2)),
        }
        if world == 1 and not args.no_cpu:
            import oracle
            threads = os.cpu_count() or 1
            ref = oracle.reference_or_none() if wl["pc"] == "sor" else None
            if ref is not None:
                ref.set_threads(threads)
                st, it, _, _, sec = getattr(ref, wl["solver"])(rp, ci, v, b, np.zeros(n), tol,
                                                               20000, precond=2)
                out["cpu_baseline"] = {"value": round(1.0 / sec, 4), "unit": "solves/s",
                                       "cores": threads, "kind": "reference",
                                       "sample": f"1 full solve ({it} iterations)"}
            else:
                # the reference has no CPU IC / ILU (ic.cpp, ilu.cpp throw "on CPU
                # does not impl."): the oracle's sequential restatement
                rs = oracle.restatement()
                t0 = time.perf_counter()
                st, it, _, _ = getattr(rs, wl["solver"])(rp, ci, v, b, np.zeros(n), tol, 20000,
                                                         precond=kind)
                sec = time.perf_counter() - t0
                out["cpu_baseline"] = {"value": round(1.0 / sec, 4), "unit": "solves/s",
                                       "cores": 1, "kind": "port",
                                       "sample": f"1 full solve ({it} iterations), the oracle's "
                                                 "sequential C restatement"}
        if cl:
            out["clocks"] = cl
    pc.close()
    A.close()
    h.close()
    return out


# ----------------------------------------------------------- batch leg
def batch_inputs(wl):
    """Systems, right-hand sides b = A x_true (x_true ~ U[-1,1], seed 3 + k)
    and per-system absolute tolerances 1e-8 * ||b_k||."""
    from monolish_b200 import workloads as W
    count = wl.get("size") or wl["count"]
    systems = W.diffusion_batch(count, seed=3)
    bs = [host_matvec(rp, ci, v, W.uniform_mt(len(rp) - 1, -1.0, 1.0, 3 + k))
          for k, (rp, ci, v) in enumerate(systems)]
    tol = np.array([1e-8 * np.linalg.norm(b) for b in bs])
    return systems, bs, tol


def cpu_reference_batch(systems, bs, tol, every, threads):
    """The reference's CG (Jacobi) on every `every`-th system; returns the
    extrapolated seconds for the whole batch and the sample size."""
    import oracle
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    ref = oracle.reference_or_none()
    if ref is None:
        return None, 0, "port"
    ref.set_threads(threads)
    idx = list(range(0, len(systems), every))
    total = 0.0
    for k in idx:
        rp, ci, v = systems[k]
        st, it, res, x, sec = ref.cg(rp, ci, v, bs[k], np.zeros(len(bs[k])), float(tol[k]), 20000)
        total += sec
    return total * len(systems) / len(idx), len(idx), "reference"


def run_batch(args, wl, rank, world, local):
    import torch
    import torch.distributed as dist
    from monolish_b200 import device as D

    torch.cuda.set_device(local)
    systems, bs, tol = batch_inputs(wl)
    count_total = len(systems)
    if world > 1:
        # the systems are independent: each rank solves its share (placed by
        # footprint), no collective on the data path
        from monolish_b200.shard import footprint_bytes, shard_by_footprint
        nk = np.array([len(rp) - 1 for rp, _, _ in systems], np.int64)
        zk = np.array([int(rp[-1]) for rp, _, _ in systems], np.int64)
        mine = shard_by_footprint(footprint_bytes(nk, zk), world)[rank]
        systems = [systems[i] for i in mine]
        bs = [bs[i] for i in mine]
        tol = tol[mine]
    count = len(systems)
    h = D.Handle()
    B = D.Batch(h, systems)
    b_all = np.concatenate(bs)
    db = torch.from_numpy(b_all).cuda()
    dx = torch.zeros_like(db)
    stream = torch.cuda.current_stream()
    mixed = args.precision == "mixed"
    inner_tol = 1e-2 if args.inner_tol is None else args.inner_tol

    def batch_solve():
        if mixed:
            return B.solve_mixed(db, dx, tol, 20000, inner_tol=inner_tol)
        return B.solve("cg", db, dx, tol, 20000)

    # untimed: the autotuner picks the rows-per-CTA cap (bins and cluster
    # shapes) per solve kind by timing full solves; x is left as it was
    tuned = {}
    for kind in (["mixed", "cg"] if mixed else ["cg"]):
        cap, best_s = B.autotune(kind, db, dx, tol, 20000, inner_tol=inner_tol)
        tuned[kind] = {"rows_per_cta_cap": cap, "groups": B.info(kind)[1],
                       "best_solve_ms": round(best_s * 1e3, 3)}
    for _ in range(args.warmup):
        dx.zero_()
        status, iters, resid = batch_solve()
    n_launch = B.info("mixed" if mixed else "cg")[1]  # one launch per group
    batch_traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "batch_cg.traffic.json")) as f:
            batch_traffic = json.load(f).get("dram_bytes_per_step")
    except (OSError, ValueError):
        pass
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        dx.zero_()
        status, iters, resid = batch_solve()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cl = clocks.stop()
    x_all = dx.cpu().numpy()
    # end to end: b from pinned host memory, x back, per batch solve
    hb = torch.from_numpy(b_all).pin_memory()
    hx = torch.empty_like(hb).pin_memory()
    e0.record(stream)
    for _ in range(max(1, min(args.steps, 3))):
        db.copy_(hb, non_blocking=True)
        dx.zero_()
        batch_solve()
        hx.copy_(dx, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / max(1, min(args.steps, 3))
    # mixed: the same batch in plain FP64, timed the same way
    fp64_ms, fp64_iters = None, None
    if mixed:
        for _ in range(2):
            dx.zero_()
            B.solve("cg", db, dx, tol, 20000)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            dx.zero_()
            _, it64, _ = B.solve("cg", db, dx, tol, 20000)
        e1.record(stream)
        torch.cuda.synchronize()
        fp64_ms = e0.elapsed_time(e1) / args.steps
        fp64_iters = int(np.asarray(it64).sum())
        dx.zero_()
        batch_solve()
        x_all = dx.cpu().numpy()
    # the comparison: a loop of single plain FP64 solves (mlsh_cg_solve per
    # system, its default engine), device time over the whole loop
    loop_ms = None
    loop_iters = None
    if not args.quick:
        plans = [D.Crs(h, len(rp) - 1, len(rp) - 1, rp, ci, v, validate=False)
                 for rp, ci, v in systems]
        dbs = [torch.from_numpy(b).cuda() for b in bs]
        dxs = [torch.zeros_like(d) for d in dbs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        loop_iters = []
        for k in range(count):
            r = D.cg_solve(plans[k], dbs[k], dxs[k], float(tol[k]), 20000)
            loop_iters.append(r.iters)
        e1.record(stream)
        torch.cuda.synchronize()
        loop_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
        for A in plans:
            A.close()
    if world > 1:
        t = torch.tensor([ms, e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])
    out = None
    if rank == 0:
        xs = np.split(x_all, np.cumsum([len(b) for b in bs])[:-1])
        sample = list(range(0, count, max(1, count // 32)))
        worst = max(true_relres(*systems[k], bs[k], xs[k]) for k in sample)
        per_step_s = ms / 1e3 / args.steps
        value = count_total / per_step_s
        rows = int(sum(len(b) for b in bs))
        nnz = int(sum(int(rp[-1]) for rp, _, _ in systems))
        iters = np.asarray(iters)
        # algorithmic bytes of the fused CG iteration, summed over systems
        vb, xb = (4, 4) if mixed else (8, 8)  # value / vector bytes of the iteration
        bytes_all = float(sum(it * ((int(systems[k][0][-1]) * (vb + 4) + (len(bs[k]) + 1) * 4)
                                    + 13 * len(bs[k]) * xb) for k, it in enumerate(iters)))
        peak, peak_kind = measured_peak()
        out = {
            "metric": METRIC_BATCH, "value": round(value, 2), "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 iteration / f64 refresh" if mixed else "f64",
            "data": "synthetic (seeded generators)",
            "config": {"workload": f"{count_total} variable-coefficient 2D diffusion systems, n "
                                   "log-uniform in [1e3, 1e5] (seed 3), Jacobi-CG to 1e-8 "
                                   "relative residual, " +
                                   (f"mixed FP32/FP64 (refresh every {inner_tol:g})" if mixed
                                    else "FP64") + ", one launch per cluster-size group",
                       "systems": count_total, "systems_on_rank0": count,
                       "rows_on_rank0": rows, "nnz_on_rank0": nnz,
                       "iters_total": int(iters.sum()), "iters_max": int(iters.max()),
                       "all_converged": bool((np.asarray(status) == 0).all()),
                       "worst_true_rel_residual_sampled": worst,
                       "autotuned": tuned,
                       "parallelism": f"systems sharded by footprint over {world} GPU(s)"},
            "e2e": {"value": round(count_total / (e2e_ms / 1e3), 2), "unit": "solves/s",
                    "h2d_bytes_per_step": b_all.nbytes, "d2h_bytes_per_step": b_all.nbytes},
            "roofline": {"bound": "hbm", "achieved": round(bytes_all / per_step_s / 1e9, 1),
                         "peak": peak, "unit": "GB/s",
                         "frac": round(bytes_all / per_step_s / 1e9 / peak, 4),
                         "peak_kind": peak_kind,
                         "traffic": batch_traffic if (not mixed and count_total == 2048) else None,
                         "traffic_unit": "DRAM bytes per batch solve (all its launches)",
                         "note": "fused-CG algorithmic bytes summed over systems / batch time; "
                                 "the iteration vectors live in the clusters' shared memory and "
                                 "each system's matrix stays in L2, so DRAM moves about 5 % of "
                                 "these bytes: a throughput figure, not a fraction of HBM "
                                 "traffic (the batch is bound by its largest systems' "
                                 "iteration latency)"},
            "gpu_launches": args.steps * n_launch,
        }
        if loop_ms is not None:
            out["loop_of_single_solves"] = {
                "value": round(count / (loop_ms / 1e3), 2), "unit": "solves/s",
                "speedup_of_batch": round((count / per_step_s) / (count / (loop_ms / 1e3)), 2)}
            if not mixed:
                out["loop_of_single_solves"]["iters_match"] = bool(
                    np.array_equal(np.asarray(loop_iters), iters))
        if mixed and fp64_ms is not None:
            out["fp64_batch"] = {"value": round(count / (fp64_ms / 1e3), 2), "unit": "solves/s",
                                 "iters_total": fp64_iters,
                                 "speedup_of_mixed": round(fp64_ms / (per_step_s * 1e3), 3)}
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            sec, ns, kind = cpu_reference_batch(systems, bs, tol, max(1, count // 16), threads)
            if sec:
                out["cpu_baseline"] = {"value": round(count / sec, 3), "unit": "solves/s",
                                       "cores": threads, "kind": kind,
                                       "sample": f"{ns} of {count} systems (every "
                                                 f"{max(1, count // 16)}th), time scaled to "
                                                 "the whole batch"}
        if cl:
            out["clocks"] = cl
    B.close()
    h.close()
    return out


# ---------------------------------------------------------- serving leg
METRIC_SERVE = "served solves/s (open-loop Poisson arrivals), p50/p99 latency"
# a stream per offered rate: about --serve-seconds of arrivals, within these
# bounds (20,000 distinct requests of the stream's size mix would need
# about 440 GB of host matrices, so the streams cycle through a pool)
SERVE_MIN_REQUESTS = 100
SERVE_MAX_REQUESTS = 2000
# inner tolerance of the stream's mixed-precision requests (the stream's
# recipe leaves it open; 1e-2 keeps the FP32 iterations well above their
# attainable accuracy, see the mixed-precision sweep of bicgstab_convdiff)
SERVE_INNER_TOL = 1e-2


def serve_requests(count, seed=4, lo=1e3, hi=2e6):
    """The request stream: per request a family (CG on 2D or 3D
    variable-coefficient diffusion, or BiCGSTAB on upwind
    convection-diffusion with Peclet ~ U[0,20]), a size log-uniform in
    [lo, hi], tol 1e-8 or 1e-10 (relative to ||b||) and plain FP64 or mixed
    precision, each chosen uniformly (numpy PCG64(seed)); b = A x_true with
    x_true ~ U[-1,1]."""
    from monolish_b200 import workloads as W
    rng = np.random.default_rng(seed)
    sizes = W.loguniform_sizes(count, lo, hi, seed)
    reqs = []
    for k in range(count):
        fam = int(rng.integers(3))
        rel = (1e-8, 1e-10)[int(rng.integers(2))]
        prec = ("fp64", "mixed")[int(rng.integers(2))]
        pe = float(rng.uniform(0.0, 20.0))
        n = int(sizes[k])
        if fam == 0:
            nx, ny = W.grid2d_for(n)
            _, rp, ci, v = W.vardiff2d(nx, ny, seed, k)
            kind = "cg"
        elif fam == 1:
            m = max(2, int(round(n ** (1.0 / 3.0))))
            nz = max(1, -(-n // (m * m)))
            _, rp, ci, v = W.vardiff3d(m, m, nz, seed, k)
            kind = "cg"
        else:
            m = max(2, int(round(n ** (1.0 / 3.0))))
            _, rp, ci, v = W.convdiff3d(m, peclet=pe)
            kind = "bicgstab"
        xt = W.uniform_fast(len(rp) - 1, -1.0, 1.0, 1000 * seed + k)
        b = host_matvec(rp, ci, v, xt)
        reqs.append(dict(kind=kind, family=("cg2d", "cg3d", "bicgstab")[fam], precision=prec,
                         rel=rel, rp=rp, ci=ci, v=v, b=b,
                         tol=rel * float(np.linalg.norm(b))))
    return reqs


def serve_stream(D, reqs, rate, budget, lanes, seed, maxiter, start=None):
    """Submit `reqs` at Poisson arrival times (rate req/s) from a producer
    thread; returns per-request results and (serving-kernel launches, lane
    solves) during the stream.  `start`, if given, is called after the
    warm-up and before the first arrival (a barrier across ranks)."""
    import threading
    if not reqs:  # a rank with no share still takes the barrier
        if start is not None:
            start()
        return [], (0, 0)
    srv = D.Server(budget, lanes)
    # warm-up: the smallest request of each kind and precision (serving
    # kernels, lanes, their first launches); not part of the stream
    warm = {}
    for q in sorted(reqs, key=lambda q: len(q["b"])):
        warm.setdefault((q["kind"], q["precision"]), q)
    for q in warm.values():
        srv.wait(srv.submit(q["kind"], q["rp"], q["ci"], q["v"], q["b"], q["tol"], maxiter,
                            precision=q["precision"], inner_tol=SERVE_INNER_TOL))
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, len(reqs))
    arrivals = np.cumsum(gaps) - gaps[0]
    ids = [None] * len(reqs)

    def producer():
        t0 = time.perf_counter()
        for k, q in enumerate(reqs):
            dt = t0 + arrivals[k] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids[k] = srv.submit(q["kind"], q["rp"], q["ci"], q["v"], q["b"], q["tol"], maxiter,
                                precision=q["precision"], inner_tol=SERVE_INNER_TOL)

    if start is not None:
        start()
    l0, s0 = srv.stats()
    th = threading.Thread(target=producer)
    th.start()
    th.join()
    res = [srv.wait(i) for i in ids]
    l1, s1 = srv.stats()
    srv.close()
    return res, (l1 - l0, s1 - s0)


def serve_loop_of_single_solves(D, h, reqs, maxiter):
    """The comparison: requests one after another through the single-solve
    entry points (upload, plan, plain FP64 solve, download); wall time."""
    import torch
    t0 = time.perf_counter()
    iters = []
    for q in reqs:
        n = len(q["b"])
        A = D.Crs(h, n, n, q["rp"], q["ci"], q["v"], validate=False)
        db = torch.from_numpy(q["b"]).cuda()
        dx = torch.zeros_like(db)
        fn = D.cg_solve if q["kind"] == "cg" else D.bicgstab_solve
        r = fn(A, db, dx, q["tol"], maxiter)
        dx.cpu()
        A.close()
        iters.append(r.iters)
    return time.perf_counter() - t0, iters


def solve_bytes(q, iters):
    """Algorithmic HBM bytes of a Jacobi-CG / BiCGSTAB solve (fused minimum
    per iteration: one SpMV pass (two for BiCGSTAB) plus the vector traffic)."""
    n = len(q["b"])
    nnz = int(q["rp"][-1])
    sp = nnz * 12 + (n + 1) * 4
    return iters * (sp + 13 * n * 8 if q["kind"] == "cg" else 2 * sp + 22 * n * 8)


def gather_parts(obj, world):
    """Every rank's `obj` (a small dict of host results), in rank order;
    a reporting exchange after the timed region, not part of the solves."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def serve_entry(rate, parts):
    """One sweep entry of the whole job from the ranks' stream results:
    latencies pooled, makespan the longest rank's."""
    lat = np.concatenate([np.asarray(p["lat"], np.float64) for p in parts])
    span = max(p["span"] for p in parts)
    return {"rate_req_s": rate, "solves_per_s": round(len(lat) / span, 2),
            "p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 2),
            "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 2),
            "makespan_s": round(span, 3),
            "all_converged": all(p["ok"] for p in parts),
            "ring_requests": sum(p["ring"] for p in parts),
            "lane_requests": sum(p["lane"] for p in parts)}


def run_serve(args, wl, rank, world, local):
    import torch
    from monolish_b200 import device as D
    torch.cuda.set_device(local)
    count = args.size or wl["count"]
    reqs_all = serve_requests(count, seed=4)
    reqs, start = reqs_all, None
    if world > 1:
        # requests are independent: each rank serves its share (placed by
        # footprint) as a stream of its own at its share of the arrival
        # rate; no collective on the data path, the ranks only start each
        # stream together and merge their results afterwards
        import torch.distributed as dist
        from monolish_b200.shard import footprint_bytes, shard_by_footprint
        nk = np.array([len(q["b"]) for q in reqs_all], np.int64)
        zk = np.array([int(q["rp"][-1]) for q in reqs_all], np.int64)
        mine = shard_by_footprint(footprint_bytes(nk, zk), world)[rank]
        reqs = [reqs_all[i] for i in mine]
        start = dist.barrier
    share = len(reqs) / count
    rates = [float(r) for r in args.rates.split(",")]
    budget, lanes, maxiter = int(wl["budget"]), args.lanes, 100000
    h = D.Handle()
    sweep = []
    clocks = ClockSampler(local)
    head = None

    def stream_of(rate):
        # about serve_seconds of arrivals at this rate (at least 100, at most
        # 2,000 requests), cycling through the pool of distinct requests
        total = int(min(SERVE_MAX_REQUESTS, max(SERVE_MIN_REQUESTS, rate * args.serve_seconds)))
        mine = max(1, int(round(total * share))) if reqs else 0
        return [reqs[k % len(reqs)] for k in range(mine)], total

    streamed = 0
    for k, rate in enumerate(rates):
        if k == len(rates) - 1:
            clocks.start()
        stream, total = stream_of(rate)
        streamed += total
        res, (launches, lane_solves) = serve_stream(D, stream, rate * share, budget, lanes,
                                                    40 + k + 1000 * rank, maxiter, start)
        part = {"lat": [r.t_done - r.t_submit for r in res],
                "span": (max(r.t_done for r in res) - min(r.t_submit for r in res)
                         if res else 0.0),
                "ok": all(r.status == 0 for r in res),
                "ring": sum(1 for r in res if r.path == 0),
                "lane": sum(1 for r in res if r.path == 1)}
        got = gather_parts(part, world)
        entry = serve_entry(rate, got)
        entry["requests"] = total
        sweep.append(entry)
        head = (stream, res, launches, lane_solves, entry, max(p["span"] for p in got), total)
    cl = clocks.stop()
    stream, res, launches, lane_solves, entry, span, head_total = head
    # the knee: the highest offered rate the server keeps up with (delivers
    # at least 95 % of it)
    kept = [e["rate_req_s"] for e in sweep if e["solves_per_s"] >= 0.95 * e["rate_req_s"]]
    knee = max(kept) if kept else None
    loop_s = None
    if not args.quick and world == 1:
        loop_s, _ = serve_loop_of_single_solves(D, h, reqs, maxiter)
    h.close()
    # true residual of every request, recomputed on the host in FP64
    worst_mine = max((true_relres(q["rp"], q["ci"], q["v"], q["b"], r.x) / q["rel"]
                      for q, r in zip(stream, res)), default=0.0)
    bytes_mine = float(sum(solve_bytes(q, r.iters) for q, r in zip(stream, res)
                           if q["precision"] == "fp64"))
    parts = gather_parts({"worst": worst_mine, "bytes": bytes_mine,
                          "launches": int(launches + lane_solves)}, world)
    if rank != 0:
        return None
    worst = max(p["worst"] for p in parts)
    bytes_all = sum(p["bytes"] for p in parts)
    launches_all = sum(p["launches"] for p in parts)
    reqs = reqs_all
    peak, peak_kind = measured_peak()
    head_reqs = [reqs[k % len(reqs)] for k in range(head_total)]
    h2d = int(sum(q["rp"].nbytes + q["ci"].nbytes + q["v"].nbytes + q["b"].nbytes
                  for q in head_reqs))
    d2h = int(sum(q["b"].nbytes for q in head_reqs))
    value = head_total / span
    fam = {f: sum(1 for q in reqs if q["family"] == f) for f in ("cg2d", "cg3d", "bicgstab")}
    out = {
        "metric": METRIC_SERVE, "value": round(value, 2), "unit": "solves/s",
        "n_gpus": world, "steps": 1, "warmup": args.warmup,
        "ms_per_step": round(span * 1e3, 1), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64 / f32-inner mixed",
        "data": "synthetic (seeded generators)",
        "config": {"workload": f"open-loop streams cycling through {count} distinct requests "
                               "(seed 4): CG on 2D/3D variable-coefficient diffusion or "
                               "BiCGSTAB on convection-diffusion (Peclet U[0,20]), n log-"
                               "uniform in [1e3, 2e6], tol 1e-8 or 1e-10, FP64 or mixed, "
                               f"Poisson arrivals; about {args.serve_seconds:g} s of arrivals "
                               f"per offered rate ({SERVE_MIN_REQUESTS}-{SERVE_MAX_REQUESTS} "
                               "requests)",
                   "distinct_requests": count, "requests_streamed": streamed,
                   "requests_at_headline_rate": head_total,
                   "knee_req_s": knee, "families": fam,
                   "mixed_requests": sum(1 for q in reqs if q["precision"] == "mixed"),
                   "rows_total": int(sum(len(q["b"]) for q in reqs)),
                   "memory_budget_bytes": budget, "lanes": lanes,
                   "mixed_inner_tol": SERVE_INNER_TOL,
                   "headline_rate_req_s": rates[-1],
                   "p50_ms": entry["p50_ms"], "p99_ms": entry["p99_ms"],
                   "worst_true_rel_residual_over_tol": worst,
                   "all_converged": entry["all_converged"],
                   "l2": "no flush: each request's matrix is uploaded from the host",
                   "parallelism": ("one GPU: serving-kernel rings + worker lanes" if world == 1
                                   else f"requests sharded by footprint over {world} GPUs, "
                                        "each serving its share at its share of the rate")},
        "sweep": sweep,
        "e2e": {"value": round(value, 2), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "note": "the served stream is end to end: host CRS and b in, x out"},
        "roofline": {"bound": "hbm", "achieved": round(bytes_all / span / 1e9, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(bytes_all / span / 1e9 / peak, 4), "peak_kind": peak_kind,
                     "traffic": None,
                     "note": "algorithmic solve bytes of the FP64 requests only / makespan"},
        "gpu_launches": int(launches_all),
        "gpu_launches_note": "serving-kernel launches + lane solves (a lower bound: each "
                             "lane solve launches one graph or cluster kernel at least)",
    }
    if loop_s is not None:
        out["loop_of_single_solves"] = {
            "value": round(len(reqs) / loop_s, 2), "unit": "solves/s",
            "speedup_of_server": round(value / (len(reqs) / loop_s), 2),
            "note": "same requests one at a time, plain FP64, wall time"}
    if world == 1 and not args.no_cpu:
        cb = cpu_reference_serve(reqs, seconds=20.0)
        if cb:
            out["cpu_baseline"] = cb
    if cl:
        out["clocks"] = cl
    return out


def cpu_reference_serve(reqs, seconds):
    """The reference's CPU CG / BiCGSTAB (Jacobi, plain FP64) on requests
    taken in a seeded random order until `seconds` of solve time; solves/s
    = solved / their summed time."""
    import oracle
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    ref = oracle.reference_or_none()
    if ref is None:
        return None
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    order = np.random.default_rng(99).permutation(len(reqs))
    total, done = 0.0, 0
    for k in order:
        q = reqs[k]
        st, it, res, x, sec = getattr(ref, q["kind"])(q["rp"], q["ci"], q["v"], q["b"],
                                                      np.zeros(len(q["b"])), q["tol"], 100000)
        total += sec
        done += 1
        if total > seconds:
            break
    return {"value": round(done / total, 3), "unit": "solves/s", "cores": threads,
            "kind": "reference",
            "sample": f"{done} of {len(reqs)} requests in seeded random order, plain FP64 "
                      f"(the reference has no mixed form), {total:.1f} s of solves"}


# ---------------------------------------------------------- reference arm
ORACLE_GEN_LIB = os.path.join(ROOT, "oracle", "_build", "libmlsh_gen_oracle.so")


def run_reference(args, wl, rank, world):
    if rank != 0:
        return None
    # the reference arm maps no library of the product: its inputs come from
    # the oracle-side build of the same generator source (same bytes)
    from monolish_b200 import workloads as W
    if not os.path.exists(ORACLE_GEN_LIB):
        subprocess.run(["make", "-s", "gen"], cwd=os.path.join(ROOT, "oracle"), check=True)
    W.set_library(ORACLE_GEN_LIB)
    if wl["kind"] == "serve":
        reqs = serve_requests(args.size or wl["count"], seed=4)
        cb = cpu_reference_serve(reqs, seconds=60.0)
        if cb is None:
            return {"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) "
                                                        "not present"}
        return {"metric": METRIC_SERVE, "value": cb["value"], "unit": "solves/s",
                "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded generators)", "impl": "reference",
                "config": {"workload": f"{len(reqs)}-request serving stream, solved one "
                                       "after another on the host"},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    if wl["kind"] == "batch":
        threads = os.cpu_count() or 1
        systems, bs, tol = batch_inputs(wl)
        count = len(systems)
        every = max(1, count // 16)
        sec, ns, kind = cpu_reference_batch(systems, bs, tol, every, threads)
        value = count / sec
        return {"metric": METRIC_BATCH, "value": round(value, 3), "unit": "solves/s",
                "n_gpus": world, "steps": 1, "warmup": 0,
                "ms_per_step": round(sec * 1e3, 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generators)", "impl": "reference",
                "config": {"workload": f"{count}-system diffusion batch, Jacobi-CG to 1e-8"},
                "cpu_baseline": {"value": round(value, 3), "unit": "solves/s",
                                 "cores": threads, "kind": kind,
                                 "sample": f"{ns} of {count} systems (every {every}th), time "
                                           "scaled to the whole batch"},
                "e2e": {"value": round(value, 3), "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    threads = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ.setdefault("OMP_PROC_BIND", "close")
    n, rp, ci, v, x = make_matrix(wl)
    if wl["kind"] == "precond":
        import oracle
        b = host_matvec(rp, ci, v, x)
        tol = 1e-10 * float(np.linalg.norm(b))
        ref = oracle.reference_or_none() if wl["pc"] == "sor" else None
        secs = []
        for _ in range(max(1, min(args.steps, 3))):
            if ref is not None:
                ref.set_threads(threads)
                st, it, _, _, sec = getattr(ref, wl["solver"])(rp, ci, v, b, np.zeros(n), tol,
                                                               20000, precond=2)
            else:
                rs = oracle.restatement()
                t0 = time.perf_counter()
                st, it, _, _ = getattr(rs, wl["solver"])(rp, ci, v, b, np.zeros(n), tol, 20000,
                                                         precond=PC_KIND[wl["pc"]])
                sec = time.perf_counter() - t0
            secs.append(sec)
        value = 1.0 / statistics.mean(secs)
        kind = "reference" if ref is not None else "port"
        cores = threads if ref is not None else 1
        return {"metric": METRIC_PRECOND, "value": round(value, 4), "unit": "solves/s",
                "n_gpus": world, "steps": len(secs), "warmup": 0,
                "ms_per_step": round(statistics.mean(secs) * 1e3, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generators)", "impl": "reference",
                "config": {"workload": describe(wl), "n": n, "iters": it, "status": st},
                "cpu_baseline": {"value": round(value, 4), "unit": "solves/s", "cores": cores,
                                 "kind": kind,
                                 "sample": f"{len(secs)} full solves" + (
                                     "" if ref is not None else
                                     " of the oracle's restatement (the reference has no CPU "
                                     "IC / ILU)")},
                "e2e": {"value": round(value, 4), "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    import oracle
    ref = oracle.reference_or_none()
    kind = "reference" if ref is not None else "port"
    if wl["kind"] == "spmv":
        nnz = int(rp[-1])
        vsz = 8 if wl["dtype"] == "f64" else 4
        B = spmv_bytes(n, nnz, vsz)
        if ref is not None:
            ref.set_threads(threads)
            ref.spmv(rp, ci, v, x, reps=max(1, args.warmup))
            _, mean_s, _ = ref.spmv(rp, ci, v, x, reps=args.steps)
        else:
            threads = 1
            mean_s, _, _ = cpu_reference_spmv(rp, ci, v, x, args.steps, 1)
        value = B / mean_s / 1e9
        return {"metric": METRIC_SPMV, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(mean_s * 1e3, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
                "data": "synthetic (seeded generators)", "impl": "reference",
                "config": {"workload": describe(wl), "n": n, "nnz": nnz, "bytes_per_step": B,
                           "parallelism": "host OpenMP"},
                "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                                 "kind": kind,
                                 "sample": f"{args.steps} full SpMVs (mean), {threads} threads"},
                "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    b = host_matvec(rp, ci, v, x)
    tol = 1e-10 * float(np.linalg.norm(b))
    if ref is None:
        raise SystemExit("reference CPU build missing")
    ref.set_threads(threads)
    secs = []
    for _ in range(args.steps):
        st, it, res, xr, sec = getattr(ref, wl["kind"])(rp, ci, v, b, np.zeros(n), tol, 20000)
        secs.append(sec)
    value = 1.0 / statistics.mean(secs)
    return {"metric": METRIC_SOLVE, "value": round(value, 4), "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(statistics.mean(secs) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generators)", "impl": "reference",
            "config": {"workload": describe(wl), "n": n, "iters": it, "status": st},
            "cpu_baseline": {"value": round(value, 4), "unit": "solves/s", "cores": threads,
                             "kind": kind, "sample": f"{args.steps} full solves"},
            "e2e": {"value": round(value, 4), "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def solve_records(args, rank, world, local):
    """The solves/s half of the metric, measured in the same run as the
    default SpMV line: 128x128 Jacobi-CG; 160^3 Jacobi-BiCGSTAB plain FP64
    against mixed FP32/FP64 at inner tol 1e-4; the 2,048-system batch
    (FP64 and mixed) against a loop of single plain solves.  Each record
    carries its own timing (CUDA events, warm-up 3), iterations, true
    relative residual and roofline fraction."""
    def sub(**kw):
        a = argparse.Namespace(**vars(args))
        a.size, a.engine, a.cluster_rows, a.eager, a.inner_tol = 0, "auto", 0, False, None
        a.variant, a.no_sweep, a.warmup = -1, True, 3
        for k, val in kw.items():
            setattr(a, k, val)
        return a

    def pick(o, *keys):
        return {k: o[k] for k in keys if k in o}

    recs = {}
    o = run_solve(sub(steps=20, precision="fp64"), dict(WORKLOADS["cg_poisson2d"]), rank, world,
                  local)
    if o is not None:
        recs["cg_poisson2d_128"] = dict(
            pick(o, "value", "unit", "ms_per_step", "cpu_baseline"),
            workload=o["config"]["workload"], iters=o["config"]["iters"],
            status=o["config"]["status"], true_rel_residual=o["config"]["true_rel_residual"],
            roofline_frac=o["roofline"]["frac"], gpu_launches=o["gpu_launches"])
    o = run_solve(sub(steps=5, precision="mixed"), dict(WORKLOADS["bicgstab_convdiff"]), rank,
                  world, local)
    if o is not None:
        pl = o.get("plain_fp64", {})
        recs["bicgstab_convdiff160"] = {
            "workload": o["config"]["workload"],
            "plain_fp64": dict(pl, ms_per_step=round(1e3 / pl["value"], 3) if pl else None),
            "mixed": dict(pick(o, "value", "unit", "ms_per_step"), iters=o["config"]["iters"],
                          outer_steps=o["config"]["outer_steps"],
                          inner_tol=o["config"]["inner_tol"], status=o["config"]["status"],
                          true_rel_residual=o["config"]["true_rel_residual"],
                          fp32_layout=o["config"].get("fp32_layout"),
                          roofline_frac=o["roofline"]["frac"]),
            "mixed_over_plain": pl.get("speedup_of_mixed"),
            "cpu_baseline": o.get("cpu_baseline")}
    for prec in ("fp64", "mixed"):
        o = run_batch(sub(steps=3, precision=prec, quick=(prec == "mixed"),
                          no_cpu=args.no_cpu or prec == "mixed"),
                      dict(WORKLOADS["batch_cg"]), rank, world, local)
        if o is None:
            continue
        c = o["config"]
        r = dict(pick(o, "value", "unit", "ms_per_step", "cpu_baseline"),
                 iters_total=c["iters_total"], all_converged=c["all_converged"],
                 worst_true_rel_residual_sampled=c["worst_true_rel_residual_sampled"],
                 roofline_frac=o["roofline"]["frac"])
        if prec == "fp64":
            lo = o.get("loop_of_single_solves", {})
            r["loop_of_single_solves"] = pick(lo, "value", "unit", "iters_match")
            recs["batch2048"] = {"workload": c["workload"], "fp64": r,
                                 "batch_over_loop": lo.get("speedup_of_batch")}
        elif "batch2048" in recs:
            recs["batch2048"]["mixed"] = r
            loop = recs["batch2048"]["fp64"]["loop_of_single_solves"].get("value")
            if loop:
                recs["batch2048"]["mixed_batch_over_loop"] = round(o["value"] / loop, 2)
    return recs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="spmv_poisson3d_f64")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--size", type=int, default=0,
                    help="override the grid edge (n for zipf); for small profiling cases")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="solver workloads: plain FP64 or FP32-inner/FP64-refinement")
    ap.add_argument("--engine", choices=["auto", "kernels", "cluster"], default="auto",
                    help="solve engine for the solver workloads")
    ap.add_argument("--cluster-rows", type=int, default=0,
                    help="cluster engine: rows per CTA (0 = auto)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="SpMV kernel variant (default: autotuned per matrix)")
    ap.add_argument("--rates", default="10,30,60,100,500,2000,5000",
                    help="serve_stream: arrival rates (req/s); the last one is the headline")
    ap.add_argument("--serve-seconds", type=float, default=15.0,
                    help="serve_stream: seconds of arrivals per offered rate")
    ap.add_argument("--lanes", type=int, default=4, help="serve_stream: worker lanes")
    ap.add_argument("--inner-tol", type=float, default=None,
                    help="mixed precision: inner tolerance / FP64 update threshold "
                         "(default 1e-4 for the single solves, 1e-2 for the batch)")
    ap.add_argument("--eager", action="store_true",
                    help="solver workloads: launch iterations one by one instead of a graph "
                         "(kernel-level profiling)")
    ap.add_argument("--no-solves", action="store_true",
                    help="default SpMV workload: skip the solves/s records (CG 128^2, "
                         "BiCGSTAB 160^3 plain vs mixed, 2,048-system batch vs loop)")
    ap.add_argument("--quick", action="store_true",
                    help="timed steps only: no clock soak, no e2e, no CPU leg (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.quick:
        args.no_cpu = True
    rank, world, local = env_rank()
    wl = dict(WORKLOADS[args.workload])
    if args.size:
        wl["size"] = args.size
    if args.impl == "reference":
        out = run_reference(args, wl, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    try:
        if wl["kind"] == "spmv":
            out = run_spmv(args, wl, rank, world, local)
            if (args.workload == "spmv_poisson3d_f64" and not args.size and not args.quick
                    and not args.no_solves):
                recs = solve_records(args, rank, world, local)
                if out is not None:
                    out["solves"] = recs
        elif wl["kind"] == "batch":
            out = run_batch(args, wl, rank, world, local)
        elif wl["kind"] == "serve":
            out = run_serve(args, wl, rank, world, local)
        elif wl["kind"] == "precond":
            out = run_precond(args, wl, rank, world, local)
        else:
            out = run_solve(args, wl, rank, world, local)
    finally:
        if world > 1:
            dist.destroy_process_group()
    if out is not None:
        rl = out.get("roofline")
        if isinstance(rl, dict) and rl.get("unit") == "GB/s" and rl.get("achieved"):
            # beside the measured copy bandwidth: the nominal 8 TB/s HBM3e figure
            rl["frac_of_nominal_8tbs"] = round(float(rl["achieved"]) / NOMINAL_HBM_GBS, 4)
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
