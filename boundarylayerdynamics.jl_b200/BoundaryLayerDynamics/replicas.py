"""Multi-GPU layout: independent replicas, no data-path collective.

A single member is not sharded (one member of the largest workload fits one
GPU's HBM many times over).  With N GPUs, one process per GPU runs its own
members: the DNS benchmark runs one member per rank, an ensemble splits each
size class's members across the ranks, and a served stream can be split by
request.  The only collectives are on the host side of the measurement: the
max over ranks of the timed region and the sum of the work done.
"""

import numpy as np


def shard(n, world, rank):
    """[lo, hi) of ``rank`` in a balanced contiguous split of ``n`` items."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(int(n), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_groups(groups, world, rank):
    """The members of each ensemble group (dicts with per-member arrays ``z0`` and
    ``cs``) that ``rank`` runs; groups left empty on this rank are dropped."""
    out = []
    for g in groups:
        lo, hi = shard(len(g["z0"]), world, rank)
        if hi > lo:
            out.append(dict(g, z0=np.asarray(g["z0"])[lo:hi], cs=np.asarray(g["cs"])[lo:hi]))
    return out


def reduce_max(x, dist=None, device=None):
    """Max of a float over all ranks (``dist`` = torch.distributed, or None for one rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x, dist=None, device=None):
    """Sum of a float over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units, seconds, dist=None, device=None):
    """Units processed by all ranks divided by the slowest rank's time."""
    return reduce_sum(units, dist, device) / reduce_max(seconds, dist, device)
