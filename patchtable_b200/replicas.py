"""Replica runs over several GPUs of one node: one process per GPU, launched by torchrun.

The query path shards without any exchange: query patches are independent given the table and
separate images need nothing from each other, so every rank builds its own table and answers its
own queries -- the same workload on every rank (replicas), or its share of a set of images
(shard_by_cost) when the images are the work.  The only collective steps are the host-side agreements of a run -- a barrier around
the timed region, the slowest rank's time, and rank 0's choice of a setting -- which every rank
takes in the same order.  The same helpers run on CPU with the gloo backend.
"""
from __future__ import annotations

import os
from datetime import timedelta


def env():
    """(rank, world size, local rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", device=None, timeout_s: float = 300.0) -> None:
    """Joins the process group when more than one rank runs; a short timeout turns a rank that
    never arrives into an error on the others instead of a hang."""
    import torch.distributed as dist
    _, world, _ = env()
    if world > 1 and not dist.is_initialized():
        kw = {"device_id": device} if (device is not None and backend == "nccl") else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)


def _active() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier() -> None:
    import torch.distributed as dist
    if _active():
        dist.barrier()


def max_over_ranks(x: float, device="cpu") -> float:
    """The largest x of all ranks (the slowest rank's time bounds the whole job)."""
    import torch
    import torch.distributed as dist
    if not _active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def agree(x: float, device="cpu") -> float:
    """Rank 0's value of x on every rank (settings chosen by measurement must match)."""
    import torch
    import torch.distributed as dist
    if not _active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.broadcast(t, src=0)
    return float(t.item())


def shard_by_cost(costs, world: int):
    """Splits items with the given costs (e.g. query patches per image) over `world` ranks: the
    most expensive first, each to the rank with the least total so far (ties: lowest rank), so the
    largest share exceeds the mean by less than one item.  Returns one sorted index list per rank;
    every rank computes the same split without communicating."""
    load = [0] * world
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def whole_job_rate(units_per_rank: float, seconds: float, world: int) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds


def finish() -> None:
    import torch.distributed as dist
    if _active():
        dist.barrier()
        dist.destroy_process_group()
