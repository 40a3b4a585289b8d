"""Multi-GPU placement: one process per GPU, no collective on the data path.

A single system does not shard (a 2-D block-cyclic factorization would be a
different algorithm), so several GPUs run replicas.  A batch of independent
systems shards by system: each rank factors and solves its share with the
batched solver, and only the per-system reports travel (a host-side gather
at the end).  Timings are the maximum over ranks.
"""
from __future__ import annotations

import heapq


def partition_systems(ns, world: int) -> list[list[int]]:
    """Greedy longest-processing-time split of systems (orders ns) over
    `world` ranks by factor cost n^3; deterministic (ties go to the lower
    rank, systems taken largest first, index order among equal sizes).
    Returns, per rank, the sorted list of system indices it owns."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(ns)), key=lambda i: (-int(ns[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(ns[i]) ** 3, r))
    return [sorted(s) for s in shards]


def shard_cost(ns, shard) -> float:
    return sum(float(ns[i]) ** 3 for i in shard)


def max_over_ranks(value: float, dist=None) -> float:
    """The maximum of `value` over the process group (the value itself
    without one).  Works on any backend: NCCL ranks pass a CUDA tensor,
    gloo ranks a CPU one."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def gather_by_system(local: dict, count: int, dist=None) -> list:
    """Collect {system index: result} dictionaries from every rank into one
    list ordered by system index (on every rank).  Host objects only: this is
    the end-of-batch report gather, not a data-path collective."""
    merged = dict(local)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
        merged = {}
        for p in parts:
            merged.update(p)
    if sorted(merged) != list(range(count)):
        raise RuntimeError("results missing or duplicated across ranks")
    return [merged[i] for i in range(count)]
