"""Instance sharding of batched workloads across GPUs.

A single LP is not partitioned (replicas only).  Batches of independent LPs
(the uneven multi-LP workload, family training and evaluation sets) shard
naturally: each process owns one GPU and a subset of the LPs, balanced by
nonzeros, solves it with no per-iteration communication, and the results meet
on rank 0 once at the end (torch.distributed: NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq


def partition(weights, world: int) -> list[list[int]]:
    """Longest-processing-time split: instances in decreasing weight, each to
    the currently lightest rank (ties to the lower rank); every rank's list is
    in increasing instance order.  Deterministic."""
    if world < 1:
        raise ValueError("world must be positive")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(p) for p in parts]


def gather(local: dict, group=None) -> dict | None:
    """Merge every rank's {instance: result} on rank 0 (None elsewhere)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    objs = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(local, objs, dst=0, group=group)
    if objs is None:
        return None
    merged: dict = {}
    for o in objs:
        merged.update(o)
    return merged


def max_over_ranks(values: list[float], device=None) -> list[float]:
    """Element-wise maximum of per-rank timings (all ranks get the result)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
