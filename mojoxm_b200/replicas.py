"""Replica plumbing for one-process-per-GPU runs.

The DG hot path does not exchange data between GPUs at this tier: a single
solve runs on one GPU, and independent solves (a batch, a served stream) are
partitioned across ranks with no data-path collective.  What crosses ranks is
bookkeeping only: each rank's device time (the job time is the maximum over
ranks) and its unit counts (summed).  These helpers do that over an already
initialised torch.distributed process group (gloo in tests, any backend in
runs); with no process group they act on the local values.
"""
from __future__ import annotations


def _dist():
    try:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            return dist
    except ImportError:
        pass
    return None


def rank_world():
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def shard(items, rank=None, world=None):
    """Items of this rank: every world-th item starting at rank (round robin,
    so ranks get work of similar size when items are drawn from one
    distribution)."""
    if rank is None or world is None:
        rank, world = rank_world()
    return [it for k, it in enumerate(items) if k % world == rank]


def _reduce(value, op):
    d = _dist()
    if d is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64)
    d.all_reduce(t, op=op(d))
    return float(t.item())


def max_over_ranks(value):
    return _reduce(value, lambda d: d.ReduceOp.MAX)


def sum_over_ranks(value):
    return _reduce(value, lambda d: d.ReduceOp.SUM)
