"""Replica placement of independent jobs over the GPUs of one node (one process per GPU).

A job never spans GPUs: rank r of N takes jobs r, r + N, r + 2N, ... of the stream and runs them on its own
GPU (its own mycel_server). Nothing crosses between GPUs while the jobs run; at the end the ranks exchange
their per-job latencies and iteration counts once (torch.distributed, any backend) so that every rank can
report the whole job's p50/p99 latency and aggregate SIMP iterations/s.
"""
from __future__ import annotations

import math
from typing import List, Sequence


def partition(items: Sequence, rank: int, world: int) -> list:
    """Round-robin share of ``items`` for ``rank`` of ``world`` (arrival order kept within a share)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in [0, world)")
    return list(items[rank::world])


def percentile(values: Sequence[float], q: float) -> float:
    """Nearest-rank percentile (the serving loop's own definition)."""
    v = sorted(values)
    if not v:
        return 0.0
    k = min(max(int(math.ceil(q * len(v))), 1), len(v))
    return v[k - 1]


def merge(local: dict, group=None) -> dict:
    """Combine per-rank serving results: ``local`` holds ``latencies`` (s, completed jobs), ``simp_iterations``,
    ``first_submit_s`` and ``last_finish_s`` on a clock shared by the ranks (seconds since a common start).
    Returns the whole job's p50/p99 latency and aggregate SIMP iter/s (all ranks get the same result)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    parts: List[dict] = [None] * world
    if world > 1:
        dist.all_gather_object(parts, local, group=group)
    else:
        parts = [local]
    lat = [x for p in parts for x in p["latencies"]]
    iters = sum(p["simp_iterations"] for p in parts)
    first = min(p["first_submit_s"] for p in parts)
    last = max(p["last_finish_s"] for p in parts)
    span = last - first
    return {"ranks": world, "completed": len(lat), "simp_iterations": iters,
            "simp_iter_s": iters / span if span > 0 else None,
            "p50_latency_s": percentile(lat, 0.50), "p99_latency_s": percentile(lat, 0.99)}
