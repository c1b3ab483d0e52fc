"""Multi-GPU plumbing: one process per GPU, samples sharded across ranks.

Samples are independent (the reference fans them out with no shared state,
src/main.rs:4648-4697), so the data path has no collective: each rank denoises
its own samples on its own GPU. The only cross-rank traffic is the timing and
counter reduction after a timed region (max of seconds, sum of compares).

One large sample can instead span the ranks (``dada_uniques_sharded``): each
compare call is split by uniques and its stored comps are all-gathered
(``torch_gather``), the one exchange step of that path.
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


def torch_gather(group=None, device=None):
    """The all-gather a sharded run (``dada_uniques_sharded``) exchanges its
    compare results through: torch.distributed over ``group``. The records
    are host memory, so a gloo group (``device`` None) needs no device copy;
    with ``device`` a CUDA device they go through NCCL. Give the process
    group a timeout: a rank that has gone then ends the others' exchange
    with an error instead of a wait."""
    import numpy as np
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)

    def gather(block):
        t = torch.from_numpy(np.ascontiguousarray(block, np.uint8))
        if device is not None:
            t = t.to(device)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        return torch.cat(parts).cpu().numpy()

    return gather


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


class RequestRouter:
    """Least-loaded routing of service requests over devices: a request goes
    to the device with the least outstanding work (sum of uniques x length of
    its requests not yet collected), ties to the lower device index. Requests
    are independent samples, so nothing is exchanged between devices."""

    def __init__(self, ndevices: int):
        self.load = [0] * ndevices
        self.owner = {}

    def assign(self, key, work: int) -> int:
        d = min(range(len(self.load)), key=lambda q: (self.load[q], q))
        self.load[d] += int(work)
        self.owner[key] = (d, int(work))
        return d

    def release(self, key) -> int:
        d, work = self.owner.pop(key)
        self.load[d] -= work
        return d


class MultiDeviceService:
    """One DenoiseService per device behind one submit/wait interface (the
    denoising service sharded over the GPUs of one node). ``submit`` returns a
    ticket of this object; results are each device's, so identical to
    ``dada_uniques`` on that sample."""

    def __init__(self, err, ncol, params=None, devices=(0,), hbm_budget: int = 0):
        import dada2_b200 as D

        self.devices = list(devices)
        self.services = [D.DenoiseService(err, ncol, params, device=d, hbm_budget=hbm_budget) for d in self.devices]
        self.router = RequestRouter(len(self.devices))
        self.tickets = {}
        self.next = 1

    def submit(self, seqs=None, abund=None, quals=None, prior=None, packed=None) -> int:
        import dada2_b200 as D

        pk = packed if packed is not None else D.pack_sample(seqs, abund, quals, prior)
        t = self.next
        self.next += 1
        d = self.router.assign(t, int(pk[0].size))  # sequence bytes = uniques x length
        self.tickets[t] = (d, self.services[d].submit(packed=pk))
        return t

    def wait(self, ticket: int, read_result: bool = True):
        d, inner = self.tickets.pop(ticket)
        try:
            return self.services[d].wait(inner, read_result=read_result)
        finally:
            self.router.release(ticket)

    def close(self):
        for s in self.services:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
