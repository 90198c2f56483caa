"""Replica plumbing for running the solve path on several GPUs of one node.

The path shards by request: every solve is independent, so N GPUs run N
replicas with no collective on the data path.  What the ranks share is
(i) the routing of requests, so that requests with the same interaction
tensor (grid, d, lambda, nback, period, method) always land on the GPU that
already holds it, and (ii) the timing reduction: a multi-GPU figure is the
work of all ranks divided by the slowest rank's time.

Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import hashlib
import os


def env_rank():
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def tensor_key(req) -> tuple:
    """The identity of a request's interaction tensor (what the server caches)."""
    periodic = req.MAXm > 0 or req.MAXn > 0
    return (tuple(int(v) for v in req.shape), float(req.d), float(req.lam), float(req.nback),
            int(req.MAXm), int(req.MAXn), float(req.Lm) if periodic else 0.0, float(req.Ln) if periodic else 0.0,
            req.method)


def route(req, world: int) -> int:
    """Rank that serves `req`: a stable hash of its tensor key (the same on
    every rank and every run, unlike Python's salted hash)."""
    if world <= 1:
        return 0
    h = hashlib.blake2b(repr(tensor_key(req)).encode(), digest_size=8).digest()
    return int.from_bytes(h, "little") % world


def shard(requests, rank: int, world: int):
    """This rank's share of a request stream, in arrival order."""
    return [r for r in requests if route(r, world) == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Largest `value` over all ranks of the default process group (the
    value itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
