"""Replica parallelism: one independent backend per GPU, no collective on the data path.

A state of up to 33 qubits fits one B200, and the units of work this backend serves (circuit
evaluations, batch samples, requests, finite-difference coordinates) are independent, so N
GPUs run N replicas, each on its share of the units. The only collectives are host-side
bookkeeping: the timing reduction (the maximum over ranks, so a job is as slow as its slowest
replica) and gathering per-rank results. Ranks come from torchrun's environment variables.
"""
from __future__ import annotations

import os


def rank_info():
    """(rank, world size, local rank) from RANK / WORLD_SIZE / LOCAL_RANK (single process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank, world):
    """This rank's share of independent work units: every world-th unit from `rank` on."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in 0..world-1")
    return list(items)[rank::world]


def max_over_ranks(value: float, device="cpu") -> float:
    """The maximum of a per-rank value (e.g. a device-timed duration) over all ranks."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local):
    """Every rank's list of results, concatenated in rank order (all ranks receive it)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(local))
    return [x for p in parts for x in p]


def aggregate_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank / seconds_max
