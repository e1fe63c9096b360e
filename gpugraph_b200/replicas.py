"""Bookkeeping for runs on several GPUs of one node.

The batched traversals shard by source or by graph with no exchange between
GPUs, so a multi-GPU run is N independent replicas (one process per GPU), each
working on its own disjoint share of the units: its own block of 64 seeded BFS
sources, its own slice of the many-graph batch. torch.distributed is used only
around the data path: the barrier before and after the timed region, the
slowest rank's time and the sum of the units processed. These helpers work with
any initialised process group (NCCL on GPUs, gloo on CPU in the tests) and are
no-ops on a single process.
"""
from __future__ import annotations

import numpy as np


def world_size() -> int:
    import torch.distributed as dist

    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def rank() -> int:
    import torch.distributed as dist

    return dist.get_rank() if dist.is_available() and dist.is_initialized() else 0


def barrier() -> None:
    import torch.distributed as dist

    if world_size() > 1:
        dist.barrier()


def _reduce(value: float, op: str, device: str) -> float:
    if world_size() == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device: str = "cpu") -> float:
    """The largest `value` over all ranks (every rank must call it, in the same order)."""
    return _reduce(value, "max", device)


def sum_over_ranks(value: float, device: str = "cpu") -> float:
    """The sum of `value` over all ranks (every rank must call it, in the same order)."""
    return _reduce(value, "sum", device)


def aggregate_rate(units_this_rank: float, seconds: float, device: str = "cpu") -> tuple[float, float]:
    """Whole-job rate of N replicas: the units all ranks processed divided by the
    slowest rank's time. Returns (rate, slowest seconds)."""
    slowest = max_over_ranks(seconds, device)
    return sum_over_ranks(units_this_rank, device) / slowest, slowest


def shard_bounds(n_units: int, rank_: int, world: int) -> tuple[int, int]:
    """[begin, end) of rank `rank_`'s contiguous share of n_units (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank_ < world:
        raise ValueError("bad rank/world")
    q, r = divmod(n_units, world)
    b = rank_ * q + min(rank_, r)
    return b, b + q + (1 if rank_ < r else 0)


def shard(units, rank_: int | None = None, world: int | None = None):
    """This rank's contiguous share of a sequence of independent units (graphs, sources)."""
    rank_ = rank() if rank_ is None else rank_
    world = world_size() if world is None else world
    b, e = shard_bounds(len(units), rank_, world)
    return units[b:e]


def seeded_sources(row_offsets, n: int, seed: int = 1) -> np.ndarray:
    """n distinct seeded vertices with out-degree > 0, ascending."""
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(np.diff(np.asarray(row_offsets)) > 0)
    return np.sort(rng.choice(cand, size=n, replace=False)).astype(np.int32)


def source_block(row_offsets, per_rank: int, rank_: int | None = None, world: int | None = None,
                 seed: int = 1) -> np.ndarray:
    """This rank's own block of `per_rank` sources (weak scaling: every rank runs a
    full batch, and no source is run by two ranks). The job draws per_rank * world
    distinct seeded sources; with one rank this is seeded_sources(row_offsets, per_rank)."""
    rank_ = rank() if rank_ is None else rank_
    world = world_size() if world is None else world
    if world == 1:
        return seeded_sources(row_offsets, per_rank, seed)
    allsrc = np.random.default_rng(seed).permutation(
        np.flatnonzero(np.diff(np.asarray(row_offsets)) > 0))[:per_rank * world]
    if len(allsrc) < per_rank * world:
        raise ValueError("fewer vertices with out-edges than sources asked for")
    return np.sort(allsrc[rank_ * per_rank:(rank_ + 1) * per_rank]).astype(np.int32)
