"""Multi-GPU plumbing of the replicas path.

The apply path has no exchange step between GPUs: independent matrices (batched
form) and independent requests (served form) are sharded across ranks, each rank
owns one GPU, and only timings and counts are reduced.  One process per GPU,
torch.distributed for the plumbing (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import os

import torch
import torch.distributed as dist


def world() -> tuple[int, int, int]:
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items: list, rank: int, world_size: int) -> list:
    """Round-robin share of independent work units (matrices or requests) for one rank."""
    return items[rank::world_size]


def shard_by_cost(costs: list, world_size: int) -> list[list[int]]:
    """Greedy largest-first assignment of work units (by cost) to ranks; returns index lists."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world_size
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: load[k])
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def _reduce(value: float, op) -> float:
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float) -> float:
    return _reduce(value, dist.ReduceOp.MAX)


def sum_over_ranks(value: float) -> float:
    return _reduce(value, dist.ReduceOp.SUM)
