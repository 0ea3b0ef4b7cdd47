"""Host plumbing for running the transport path on several GPUs of one node.

The path does not shard within one mesh (one-layer halo exchange and a reduction per
Krylov iteration do not pay at these sizes), so several GPUs run independent work:
replicas of one workload, or disjoint shards of a batch of independent meshes assigned
by a greedy longest-processing-time partition.  No collective touches the data path;
collectives only time the job (max over ranks) and gather per-mesh results.
"""
from __future__ import annotations

import numpy as np

from .batch import lpt_partition


def shard_of(weights, rank: int, world: int) -> list[int]:
    """Indices of the items (e.g. meshes weighted by tet count) this rank owns."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return lpt_partition(weights, world)[rank]


def max_over_ranks(value: float, device=None) -> float:
    """The job's time: the maximum of a per-rank value (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict, n_items: int) -> list | None:
    """Rank 0 receives every rank's {item index: result} merged into a list in item order."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [local[i] for i in range(n_items)]
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(local, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    missing = sorted(set(range(n_items)) - set(merged))
    if missing:
        raise RuntimeError(f"items without a result: {missing[:10]}")
    return [merged[i] for i in range(n_items)]


def imbalance(weights, parts) -> float:
    """max part load / mean part load of a partition."""
    w = np.asarray(weights, dtype=np.float64)
    loads = np.array([w[p].sum() for p in parts])
    return float(loads.max() / max(loads.mean(), 1e-300))
