"""Host logic of the multi-GPU batch path on CPU: LPT sharding of images over
ranks and the gather of results over a world-size-2 gloo process group (the
solver is replaced by a deterministic stand-in; no GPU is touched)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from artefact_b200.api import Coefficient
from artefact_b200.multigpu import job_cost, lpt_partition, solve_sharded


def _jobs(n, seed=0):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        w, h = int(rng.integers(2, 40)) * 8, int(rng.integers(2, 40)) * 8
        nch = 3 if i % 3 else 1
        coefs = [Coefficient(w, h, w // 8, h // 8, 1, 1, np.zeros(w * h, np.int16), np.ones(64, np.float32))
                 for _ in range(nch)]
        jobs.append(dict(coefs=coefs, weight=0.3, pweight=[0.001] * 3, tag=i))
    return jobs


def _fake_solve(jobs):
    return [np.full(4, j["tag"], np.float32) + job_cost(j) for j in jobs]


def test_lpt_partition_covers_each_item_once_and_balances():
    rng = np.random.default_rng(1)
    costs = rng.uniform(1, 100, 257)
    for n in (1, 2, 3, 8):
        parts = lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: the heaviest rank exceeds the mean by at most the largest item.
        assert max(loads) - sum(loads) / n <= max(costs) + 1e-9
    assert lpt_partition([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_single_rank_needs_no_group():
    jobs = _jobs(5)
    out = solve_sharded(jobs, 10, _fake_solve, rank=0, world=1)
    assert [int(o[0] - job_cost(j)) for o, j in zip(out, jobs)] == list(range(5))


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = _jobs(23, seed=3)
        out = solve_sharded(jobs, 10, _fake_solve, rank=rank, world=world)
        if rank == 0:
            q.put([int(o[0] - job_cost(j)) for o, j in zip(out, jobs)])
        else:
            q.put(out)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_gather_over_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = [r for r in res if r is not None]
    assert len(gathered) == 1 and res.count(None) == 1
    assert gathered[0] == list(range(23))
