"""Multi-GPU plumbing for walker batches: one process per GPU, walkers
sharded across ranks with no data-path collective (parameter points are
independent -- there is no exchange step inside an evaluation).  The only
collectives are the timing reduction (max over ranks) and an optional
gather of results.

Cost weights follow the contraction work per point, which grows as
n_m * n_z * n_t: 1 : 8 : 64 for the 1x / 2x / 4x grids.
"""
from __future__ import annotations

import numpy as np

DENSITY_COST = {1: 1.0, 2: 8.0, 4: 64.0}


def shard_walkers(densities, rank, world):
    """Indices of the walkers owned by `rank`: greedy cost-balanced
    assignment (largest first, ties by index) so every rank gets a similar
    share of tensor-core work.  Deterministic and identical on all ranks."""
    densities = list(densities)
    order = sorted(range(len(densities)), key=lambda i: (-DENSITY_COST.get(densities[i], 1.0), i))
    load = np.zeros(world)
    owner = np.empty(len(densities), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += DENSITY_COST.get(densities[i], 1.0)
    return [i for i in range(len(densities)) if owner[i] == rank]


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (identity without torch.distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_results(local, rank, world, device=None):
    """All-gather of per-rank result arrays (same shape on every rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or world == 1:
        return [np.asarray(local)]
    t = torch.as_tensor(np.asarray(local), dtype=torch.float64,
                        device=device if device is not None else "cpu")
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t)
    return [o.cpu().numpy() for o in outs]
