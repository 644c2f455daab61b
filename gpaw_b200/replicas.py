"""One process per GPU, independent work per process ("replicas only").

The finite-difference path has no exchange step on one grid per GPU: bands
and Poisson solves are independent units.  Multi-GPU runs therefore shard
the units across ranks and use the process group only to agree on timing
(the slowest rank's device time) and to collect results.
"""
from __future__ import annotations

import numpy as np


def shard_by_cost(costs, world, rank):
    """Indices of the units rank `rank` owns: longest-processing-time-first
    assignment of `costs` (e.g. grid points) to `world` ranks; every unit
    goes to exactly one rank and the assignment is the same on all ranks."""
    order = np.argsort(-np.asarray(costs, float), kind='stable')
    load = np.zeros(world)
    owner = np.empty(len(costs), int)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [int(i) for i in np.flatnonzero(owner == rank)]


def max_over_ranks(seconds, group=None, device=None):
    """The largest of the ranks' values (all ranks get it)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(local, group=None):
    """All ranks' (index, value) pairs, merged and sorted by index."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return sorted(local)
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, local, group=group)
    return sorted(p for part in out for p in part)
