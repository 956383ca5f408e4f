"""Multi-process paths on CPU (gloo, two ranks): the max-over-ranks clock, the barrier and
the sharding of independent solves that bench.py uses under torchrun, and a rank that
leaves before a collective (the other rank ends with an error, it does not hang)."""
from __future__ import annotations

import datetime
import os
import socket

import pytest

from inductioneq_b200 import ranks as R


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, fn, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    try:
        q.put((rank, fn(R.Ranks.from_env())))
    except Exception as e:   # reported to the parent
        q.put((rank, ("error", type(e).__name__, str(e)[:200])))


def _run(world, fn, timeout=120):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, fn, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=timeout) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def _clock(rk):
    R.init(rk, "gloo", timeout_s=30)
    R.barrier(rk)
    t = [0.25, 0.5][rk.rank]                      # this rank's device time
    t_max = R.max_over_ranks(rk, t)
    units = R.sum_over_ranks(rk, 10.0 * (rk.rank + 1))
    parts = R.partition([n ** 3 for n in (16, 96, 40, 64, 17, 80, 33)], rk.world)
    R.finish(rk)
    return t_max, units, parts


def test_max_over_ranks_barrier_and_partition_on_two_ranks():
    out = _run(2, _clock)
    assert out[0] == out[1]                       # every rank sees the same totals and split
    t_max, units, parts = out[0]
    assert t_max == 0.5 and units == 30.0
    assert sorted(parts[0] + parts[1]) == list(range(7)) and not set(parts[0]) & set(parts[1])


def _leaves(rk):
    R.init(rk, "gloo", timeout_s=5)
    if rk.rank == 1:
        return "left"                             # never reaches the collective
    import time
    t0 = time.time()
    try:
        R.barrier(rk)
        return ("no error", time.time() - t0)
    except Exception as e:
        return ("error", type(e).__name__, time.time() - t0)


def test_rank_that_leaves_ends_the_other_ranks_collective_with_an_error():
    out = _run(2, _leaves)
    assert out[1] == "left"
    assert out[0][0] == "error" and out[0][2] < 60


def test_partition_balances_and_is_deterministic():
    from inductioneq_b200.batch import rotation_batch
    specs = rotation_batch(32, seed=2026)
    costs = [n ** 3 for (n, _, _, _) in specs]
    for world in (1, 2, 4, 8):
        parts = R.partition(costs, world)
        assert parts == R.partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-first greedy: no rank above the mean by more than the largest unit
        assert max(loads) <= sum(costs) / world + max(costs)
