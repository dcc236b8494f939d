"""Placement of a batch on several GPUs (CPU only): the assignment is a
partition, balanced to within one system's footprint, identical on every
rank -- checked with two gloo ranks that compute it independently and
exchange what they got."""
import os

import numpy as np
import pytest

from monolish_b200.shard import footprint_bytes, shard_by_footprint


def test_partition_and_balance():
    rng = np.random.default_rng(3)
    n = np.exp(rng.uniform(np.log(1e3), np.log(1e5), 2048)).round().astype(np.int64)
    fp = footprint_bytes(n, 5 * n)
    for world in (1, 2, 3, 8):
        shards = shard_by_footprint(fp, world)
        allidx = np.sort(np.concatenate(shards))
        assert np.array_equal(allidx, np.arange(len(fp)))
        loads = np.array([fp[s].sum() for s in shards])
        assert loads.max() - loads.min() <= fp.max()


def test_edge_cases():
    assert [list(s) for s in shard_by_footprint([], 2)] == [[], []]
    assert [list(s) for s in shard_by_footprint([5, 5, 5], 4)] == [[0], [1], [2], []]
    with pytest.raises(ValueError):
        shard_by_footprint([1], 0)


def _rank_main(rank, world, port, sizes, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_by_footprint(footprint_bytes(sizes, 5 * sizes), world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine.tolist())
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    import torch.multiprocessing as mp
    sizes = np.array([900, 80000, 1500, 42000, 7000, 7000, 120, 65000], np.int64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    expect = shard_by_footprint(footprint_bytes(sizes, 5 * sizes), 2)
    assert [sorted(g) for g in got] == [list(e) for e in expect]
    assert sorted(got[0] + got[1]) == list(range(len(sizes)))


def _load_bench():
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _serve_rank_main(rank, world, port, out):
    """Each rank contributes a stream result of its own share; every rank
    merges the same whole-job entry."""
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench = _load_bench()
        part = ({"lat": [0.001, 0.002, 0.003], "span": 0.5, "ok": True, "ring": 2, "lane": 1}
                if rank == 0 else
                {"lat": [0.010], "span": 0.8, "ok": False, "ring": 0, "lane": 1})
        out.put((rank, bench.serve_entry(100.0, bench.gather_parts(part, world))))
    finally:
        dist.destroy_process_group()


def test_serve_results_merge_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30000 + os.getpid() % 1000
    procs = [ctx.Process(target=_serve_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got[0] == got[1]
    e = got[0]
    # 4 requests over the longest rank's makespan; latencies pooled
    assert e["solves_per_s"] == round(4 / 0.8, 2)
    assert e["makespan_s"] == 0.8
    assert e["p50_ms"] == round(float(np.percentile([1, 2, 3, 10], 50)), 2)
    assert e["all_converged"] is False
    assert (e["ring_requests"], e["lane_requests"]) == (2, 2)
