"""Multi-GPU: replicas.

Registrations are independent jobs, so N GPUs run N independent engines: one process
per GPU, each registering its own share of the jobs, with torch.distributed used only
for a barrier and for combining measurements (max of device times, gather of
per-job latencies).  There is no collective on the data path.  Within one process,
Router spreads jobs over several engines (one per visible device) by their queued
work.
"""
from __future__ import annotations

import os


def env_rank():
    """(rank, local_rank, world_size) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def shard(items, rank: int, world: int):
    """This rank's share: item k goes to rank k % world (every item exactly once)."""
    return [it for k, it in enumerate(items) if k % world == rank]


def _dev(dist):
    import torch

    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float, dist=None) -> float:
    """max of a scalar over all ranks (every rank gets it); identity without dist."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None) -> float:
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_lists(values, dist=None) -> list:
    """Concatenation of every rank's list, in rank order (every rank gets it)."""
    if dist is None:
        return list(values)
    world = dist.get_world_size()
    out = [None] * world
    dist.all_gather_object(out, list(values))
    return [v for part in out for v in part]


class Router:
    """Routes jobs over several engines (one per device) in one process: each job goes
    to the engine with the least queued work (estimated voxels of its unfinished jobs),
    ties to the lowest index.  Engines only need submit(*a, **k) -> id and
    wait(id) -> result."""

    def __init__(self, engines):
        self.engines = list(engines)
        self.load = [0.0] * len(self.engines)
        self.where = {}

    def submit(self, moving, *a, work: float | None = None, **k):
        w = float(work if work is not None else getattr(moving, "size", 1))
        e = min(range(len(self.engines)), key=lambda i: (self.load[i], i))
        jid = self.engines[e].submit(moving, *a, **k)
        self.load[e] += w
        self.where[(e, jid)] = w
        return (e, jid)

    def wait(self, handle):
        e, jid = handle
        r = self.engines[e].wait(jid)
        self.load[e] -= self.where.pop((e, jid), 0.0)
        return r
