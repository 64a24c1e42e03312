"""Sharding independent scenes or rollout requests across GPUs (one process per GPU).

Batched scenes and served requests are independent, so multi-GPU runs partition them
across ranks with no collective on the data path: each rank advances its shard with the
batched kernels, and only small per-item results (latencies, counters, optional final
states) are gathered at the end over torch.distributed (NCCL on GPUs, gloo on CPU).
"""

from __future__ import annotations

import heapq


def work_of(item) -> float:
    """Particle-substeps of a scene description or a request."""
    sc = getattr(item, "scene", item)
    return float(sc.n_particles) * float(sc.n_substeps)


def partition(items, world: int, weight=work_of) -> list[list[int]]:
    """Longest-processing-time greedy bin packing: indices of items per rank, balancing
    total weight (worst case 4/3 of the optimum)."""
    order = sorted(range(len(items)), key=lambda i: -weight(items[i]))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + weight(items[i]), r))
    for o in out:
        o.sort()
    return out


def my_shard(items, rank: int, world: int, weight=work_of):
    idx = partition(items, world, weight)[rank]
    return [items[i] for i in idx]


def gather_objects(obj, world: int):
    """All ranks' objects in rank order (identity at world 1)."""
    if world == 1:
        return [obj]
    import torch.distributed as dist

    out = [None] * world
    dist.all_gather_object(out, obj)
    return out
