"""Placement of independent systems on GPUs (the batched and served forms).

Systems are independent, so several GPUs share a batch with no collective
on the data path: each rank solves the systems assigned to it.  The
assignment balances device memory footprint (a proxy for solve work on
these bandwidth-bound solvers) with the longest-processing-time rule:
systems in decreasing footprint order, each to the rank holding the least
so far (ties to the lowest rank).  Every rank computes the same assignment
from the same sizes, so nothing has to be exchanged.
"""
from __future__ import annotations

import numpy as np


def footprint_bytes(n_rows, nnz, value_bytes=8, work_vectors=6):
    """Device bytes of one CRS system with its solver vectors."""
    n_rows = np.asarray(n_rows, np.int64)
    nnz = np.asarray(nnz, np.int64)
    return nnz * (value_bytes + 4) + (n_rows + 1) * 4 + work_vectors * n_rows * value_bytes


def shard_by_footprint(footprints, world):
    """Indices of the systems each of `world` ranks solves (ascending per
    rank); the union is every system exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    fp = np.asarray(footprints, np.int64)
    order = np.argsort(-fp, kind="stable")
    load = np.zeros(world, np.int64)
    owner = np.empty(len(fp), np.int64)
    for k in order:
        r = int(np.argmin(load))  # first minimum: the lowest rank on ties
        owner[k] = r
        load[r] += fp[k]
    return [np.flatnonzero(owner == r) for r in range(world)]
