"""Independent replicas across GPUs (one process per GPU).

The random-field path has no exchange step on one GPU per sample: tiles are
blended in device memory and realisations are independent.  Several GPUs
therefore run independent replicas; the only cross-rank operations are the
partition of an ensemble's realisations, the timing reduction (the slowest
rank defines the job's time) and gathering small per-rank results.

Realisation r of an ensemble is the same field whatever the number of ranks:
its shape, correlation length and seed depend on r alone, and rank k of W
generates the contiguous block shard(n, W, k).
"""
import numpy as np


def shard(n, world, rank):
    """Contiguous block [lo, hi) of n realisations owned by rank of world
    (sizes differ by at most one, lower ranks take the extra ones)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("invalid shard request")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def realisation_seeds(lo, hi, base=0):
    """Philox keys of realisations lo..hi-1 (key = base + realisation index)."""
    return np.arange(base + lo, base + hi, dtype=np.uint64)


def replica_seed_base(rank, stride=1000):
    """Deck seed of the replica that rank generates when every rank makes
    its own copy of the same deck sample."""
    return stride * rank


def max_over_ranks(value, dist=None, device=None):
    """The largest value over all ranks (a time: the slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device=None):
    """Sum of a per-rank count over all ranks (points generated, launches)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
