"""Multi-GPU plumbing: one process per GPU, samples sharded across ranks.

Samples are independent (the reference fans them out with no shared state,
src/main.rs:4648-4697), so the data path has no collective: each rank denoises
its own samples on its own GPU. The only cross-rank traffic is the timing and
counter reduction after a timed region (max of seconds, sum of compares).
"""
from __future__ import annotations

import os


def rank_world():
    """(rank, world, local_rank) from the torchrun environment."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def shard_samples(sizes, rank: int, world: int):
    """Indices of the samples this rank owns: greedy longest-processing-time
    assignment on `sizes` (work estimates), deterministic and disjoint."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += sizes[i]
    return [i for i in range(len(sizes)) if owner[i] == rank]


def reduce_run(seconds: float, compares: int, device=None):
    """Max of per-rank seconds and sum of per-rank compares over the default
    process group (identity when torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return seconds, compares
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    c = torch.tensor([float(compares)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(round(c.item()))
