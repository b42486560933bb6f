"""Multi-process helpers (one process per GPU, torch.distributed for the
plumbing).

The network step does not exchange data between GPUs in this build: a
multi-GPU run is replicas (independent networks, one per rank) or a sweep
batch sharded by instance (instances are independent, so no collective is
on the data path).  Gradient training is data-parallel over the trials of a
batch: each rank runs the adjoint on its own trials and one all-reduce
combines the gradients.  The other collectives are the timing reductions of
a benchmark: the slowest rank's time (max) and aggregate counts (sum).
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


def batch_slice(batch, rank, world):
    """Contiguous trial range [lo, hi) of rank's share of a data-parallel
    batch (the first batch % world ranks take one trial more)."""
    base, extra = divmod(int(batch), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def allreduce_mean_grads(tensors, n_local, n_total):
    """Combine per-rank gradients of a loss that is a mean over trials.

    Each rank holds the gradient (and loss) of the mean over its own
    n_local trials; the gradient of the mean over all n_total trials is the
    sum over ranks of (n_local / n_total) times it.  The tensors are scaled
    and all-reduced in place (one collective per tensor, in list order on
    every rank) and returned.  With one process this is the identity.
    """
    import torch.distributed as dist
    scale = float(n_local) / float(n_total)
    for t in tensors:
        t.mul_(scale)
        if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return tensors


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
