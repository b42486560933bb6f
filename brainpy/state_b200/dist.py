"""Multi-process helpers (one process per GPU, torch.distributed for the
plumbing).

The network step does not exchange data between GPUs in this build: a
multi-GPU run is replicas (independent networks, one per rank) or a sweep
batch sharded by instance (instances are independent, so no collective is
on the data path).  The only collectives are the timing reductions of a
benchmark: the slowest rank's time (max) and aggregate counts (sum).
"""
from __future__ import annotations

import os


def world_info():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base, rank):
    """Seed of rank's independent network replica."""
    return int(base) + int(rank)


def shard_instances(costs, rank, world):
    """Indices of the instances rank runs: longest-processing-time first onto
    the least-loaded rank (deterministic, so every rank computes the same
    partition without communication).  costs: per-instance work estimate."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += float(costs[i])
    return [i for i in range(len(costs)) if owner[i] == rank]


def _reduce(x, op):
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x):
    """The largest x over all ranks (the slowest rank's time)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX)


def sum_over_ranks(x):
    """The sum of x over all ranks (aggregate work)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM)
