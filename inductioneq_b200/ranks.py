"""One process per GPU: rank bookkeeping, the max-over-ranks clock and the sharding of
independent solves.

Every solve of this library runs on one GPU (the 64^3 .. 128^3 configurations fit one
B200 many times over), so several GPUs either run replicas of a workload or split a
set of independent solves between them -- neither needs a data-path collective.  The
only collectives are the barrier around a timed region and the MAX of the ranks' device
times (a job is as slow as its slowest rank), done through torch.distributed (NCCL
between GPUs, gloo on CPU).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Ranks:
    world: int
    rank: int
    local_rank: int

    @staticmethod
    def from_env() -> "Ranks":
        """RANK / LOCAL_RANK / WORLD_SIZE as torchrun sets them (a single process otherwise)."""
        return Ranks(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                     int(os.environ.get("LOCAL_RANK", "0")))


def init(ranks: Ranks, backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Join the process group (world > 1) with a bounded timeout, so that ranks that wait for
    a rank that has gone end with an error instead of hanging."""
    if ranks.world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier(ranks: Ranks) -> None:
    if ranks.world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ranks: Ranks, x: float, device=None) -> float:
    """The largest x over all ranks (every rank gets it)."""
    if ranks.world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(ranks: Ranks, x: float, device=None) -> float:
    if ranks.world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def finish(ranks: Ranks) -> None:
    if ranks.world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def partition(costs, world: int) -> list[list[int]]:
    """Split independent units (e.g. the solves of a batch, cost ~ nodes x stages) between
    `world` ranks: longest first, each to the currently lightest rank (ties to the lower
    rank), so every rank computes the same split without communicating.  Returns the unit
    indices of every rank, each list in ascending order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
