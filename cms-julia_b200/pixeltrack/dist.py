"""Event sharding over GPUs, one process per GPU (torch.distributed).

Events are independent, as the reference's stream threads are (EventProcessor.jl:43-45):
each rank reconstructs its own share of the events with its own chain and graph, and the
only collectives are scalar reductions of timings and counters. Nothing on the data path
crosses ranks.
"""
from __future__ import annotations

import datetime
import os


def world_from_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (1 process otherwise)."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def init(backend: str = "nccl", timeout_s: int = 300) -> bool:
    """Joins the process group when launched with more than one rank; returns whether it did."""
    import torch.distributed as dist
    _, world, _ = world_from_env()
    if world <= 1 or dist.is_initialized():
        return dist.is_initialized()
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return True


def shard(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of n items for rank; shares differ in size by at most one."""
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's synthetic events: distinct per rank, fixed for a given seed."""
    return seed + 7919 * rank


def _reduce(value: float, op: str, device) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device="cpu") -> float:
    """Largest value over the ranks (the job's time is its slowest rank's)."""
    return _reduce(value, "max", device)


def sum_over_ranks(value: float, device="cpu") -> float:
    return _reduce(value, "sum", device)
