"""Multi-GPU use of the solver: independent replicas and shards.

The path has no cross-instance exchange in this build: one process per GPU
solves its own mesh (replicas) or its own subset of a batch of independent
meshes (shards), and only the timing is combined (max over ranks).  There
is no data-path collective.
"""
import heapq

import numpy as np


def shard_instances(sizes, world, rank):
    """Deterministic size-balanced assignment of independent instances to
    ranks (largest first onto the least-loaded rank, ties by rank index).
    Returns the sorted instance indices of `rank`."""
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    heap = [(0, r) for r in range(world)]
    owner = np.empty(len(sizes), dtype=np.int64)
    for k in order:
        load, r = heapq.heappop(heap)
        owner[k] = r
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return sorted(int(k) for k in np.nonzero(owner == rank)[0])


def _device_for_backend():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(value):
    """Max of a float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value):
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
