"""Image-level sharding of a batch over the GPUs of one node.

A single image is one coupled problem (its TV/TGV norms couple the channels
and each channel's gradient norm couples all of its pixels every iteration),
so images are never split. A batch of images is divided between ranks (one
process per GPU, ``torch.distributed``) by the longest-processing-time rule on
pixel count; every rank solves its share as one batched launch
(``art_context_compute_batch``) and the result planes are gathered on one rank
over the process group. There is no collective on the data path: the only
exchange is the final gather of finished planes (host memory).
"""
from __future__ import annotations

import heapq
from typing import Callable, List, Optional, Sequence


def lpt_partition(costs: Sequence[float], nranks: int) -> List[List[int]]:
    """Indices of `costs` split into `nranks` lists by the longest-processing-
    time rule: items in decreasing cost (ties by index) go to the rank with the
    smallest load so far (ties by rank). Deterministic; each list is sorted."""
    if nranks < 1:
        raise ValueError("nranks must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(nranks)]
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def job_cost(job: dict) -> float:
    """Pixels a job's iterations sweep: full-resolution area times channel count."""
    coefs = job["coefs"]
    w = job.get("max_w", max(c.rounded_px_w for c in coefs))
    h = job.get("max_h", max(c.rounded_px_h for c in coefs))
    return float(w * h * job.get("nchannel", len(coefs)))


def solve_sharded(jobs: Sequence[dict], iterations: int, solve: Callable[[List[dict]], list], rank: int,
                  world: int, group=None, dst: int = 0) -> Optional[list]:
    """Solves this rank's LPT share of `jobs` with `solve` (a list of jobs ->
    a list of per-job results, e.g. ``Context.compute_batch`` bound to the
    iteration count) and gathers every result on rank `dst`, in the order of
    `jobs`. Returns that list on `dst` and None on the other ranks. With
    world == 1 no process group is needed."""
    parts = lpt_partition([job_cost(j) for j in jobs], world)
    mine = parts[rank]
    results = solve([jobs[i] for i in mine]) if mine else []
    if len(results) != len(mine):
        raise RuntimeError(f"rank {rank}: solver returned {len(results)} results for {len(mine)} jobs")
    if world == 1:
        return list(results)
    import torch.distributed as dist

    payload = list(zip(mine, results))
    gathered = [None] * world if rank == dst else None
    dist.gather_object(payload, gathered, dst=dst, group=group)
    if rank != dst:
        return None
    out: list = [None] * len(jobs)
    for part in gathered:
        for i, r in part:
            if out[i] is not None:
                raise RuntimeError(f"job {i} solved twice")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"jobs without a result: {missing[:8]}")
    return out
