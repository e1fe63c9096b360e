"""Bookkeeping for runs on several GPUs of one node.

The batched traversals shard by source or by graph with no exchange between
GPUs, so a multi-GPU run is N independent replicas (one process per GPU,
torch.distributed only for the barrier around the timed region and for the
slowest rank's time). These helpers work with any initialised process group
(NCCL on GPUs, gloo on CPU in the tests) and are no-ops on a single process.
"""
from __future__ import annotations


def world_size() -> int:
    import torch.distributed as dist

    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def barrier() -> None:
    import torch.distributed as dist

    if world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device: str = "cpu") -> float:
    """The largest `value` over all ranks (every rank must call it, in the same order)."""
    if world_size() == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, seconds: float, device: str = "cpu") -> tuple[float, float]:
    """Whole-job rate of N replicas: the units all ranks processed divided by the
    slowest rank's time. Returns (rate, slowest seconds)."""
    slowest = max_over_ranks(seconds, device)
    return world_size() * units_per_rank / slowest, slowest
