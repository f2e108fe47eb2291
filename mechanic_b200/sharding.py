"""Sharding batched scenes across GPUs (one process per GPU).

Independent scenes are the unit of work: rank r of N steps the scenes whose
cumulative body count falls in the r-th N-th of the batch total (contiguous
ranges, balanced by body count), each rank with its own batched handle.
Stepping needs no exchange; the only collective is a gather of per-rank
results at the end (torch.distributed over NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

import numpy as np


def partition(body_counts, world_size: int) -> list[list[int]]:
    """Contiguous scene ranges per rank: scene i goes to the rank whose share of the
    total holds the midpoint of i's bodies in the cumulative count."""
    counts = np.asarray(body_counts, np.int64)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    total = int(counts.sum())
    if total == 0:
        return [list(range(len(counts)))] + [[] for _ in range(world_size - 1)]
    mid = np.cumsum(counts) - counts / 2.0
    owner = np.minimum((mid * world_size / total).astype(np.int64), world_size - 1)
    return [np.nonzero(owner == r)[0].tolist() for r in range(world_size)]


def imbalance(body_counts, parts) -> float:
    """max over ranks of (rank bodies) / (total / ranks)."""
    counts = np.asarray(body_counts, np.int64)
    loads = [int(counts[p].sum()) for p in parts]
    mean = counts.sum() / len(parts)
    return max(loads) / mean if mean else 1.0


def gather_results(result: dict, group=None) -> list[dict]:
    """All ranks' result dicts, in rank order, on every rank."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return [result]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, result, group=group)
    return out


def max_over_ranks(value: float, device=None) -> float:
    """The slowest rank's time (device or CPU tensor, per backend)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
