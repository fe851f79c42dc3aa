"""Multi-GPU use of the PM step: replicas only.

A box's step has global FFTs and no data-path collective, so N GPUs run N
independent boxes (or independent subsets of an ensemble / request stream).
This module holds the host-side plumbing the benchmark and ensemble runs use
across ranks: process-group setup, a barrier, max-over-ranks timing, and the
partition of a list of boxes over ranks (greedy by predicted cost, so no
rank waits long on another).  torch.distributed is plumbing here: NCCL on
GPUs, gloo on CPU (the tests).
"""
from __future__ import annotations

import datetime
import os


class Ranks:
    """rank / world of this process, and the collectives the timing needs."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.backend = backend
        if self.world > 1:
            import torch
            import torch.distributed as dist

            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def allmax(self, v: float) -> float:
        """Max of v over ranks (the timing rule: the slowest rank's time)."""
        if self.dist is None:
            return float(v)
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(self, v: float) -> float:
        if self.dist is None:
            return float(v)
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj):
        """Every rank's obj, in rank order, on every rank (host-side results:
        latencies, per-rank summaries; no data-path use)."""
        if self.dist is None:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def box_cost(ng: int, np_side: int, nsteps: int) -> float:
    """Predicted cost of a box: particles x steps plus the grid work."""
    return float(nsteps) * (np_side ** 3 + ng ** 3)


def partition(costs, world: int):
    """Greedy longest-processing-time split of items over `world` ranks:
    returns, per rank, the list of item indices.  Deterministic (ties by
    index), so every rank computes the same split without communicating."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out
