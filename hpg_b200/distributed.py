"""Visibility sharding across ranks (one process per GPU).

Gridding is a sum over visibilities, so a batch splits into independent
shards: rank k grids its contiguous shard into its own gridder and the only
exchange is one element-wise sum of the grids and weights (an all-reduce)
when a combined image is wanted.  Degridding needs the whole model on every
rank (set it on each, or broadcast it once) and no exchange at all.

The helpers take torch.distributed process groups, so the same code runs
over NCCL between GPUs and over gloo between CPU processes (the tests).
"""
import numpy as np


def shard_bounds(n, world_size, rank):
    """[start, stop) of rank's contiguous shard of n items: sizes differ by
    at most one, the first n % world_size ranks take the larger ones."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must be in [0, world_size)")
    if n < 0:
        raise ValueError("n must be >= 0")
    base, extra = divmod(n, world_size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard(vis, world_size, rank):
    """This rank's shard of a visibility record array (a view)."""
    a, b = shard_bounds(len(vis), world_size, rank)
    return vis[a:b]


def allreduce_sum(arrays, group=None):
    """Sum numpy or torch arrays element-wise over the ranks of `group`, in
    place; returns them.  numpy arrays go through a CPU tensor (gloo), torch
    tensors stay where they are (NCCL for CUDA tensors).  Complex arrays are
    reduced as their real and imaginary parts."""
    import torch
    import torch.distributed as dist
    out = []
    for a in arrays:
        if isinstance(a, np.ndarray):
            t = torch.from_numpy(a)
            view = torch.view_as_real(t) if t.is_complex() else t
            dist.all_reduce(view, op=dist.ReduceOp.SUM, group=group)
            out.append(a)
        else:
            view = torch.view_as_real(a) if a.is_complex() else a
            dist.all_reduce(view, op=dist.ReduceOp.SUM, group=group)
            out.append(a)
    return out


def grid_sharded(grid_shard_fn, vis, group=None):
    """Grid a batch across the ranks of `group`: this rank calls
    grid_shard_fn(its shard) -> (grid, weights), then the grids and weights
    of all ranks are summed; every rank returns the combined pair."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    grid, weights = grid_shard_fn(shard(vis, world, rank))
    allreduce_sum([grid, weights], group=group)
    return grid, weights
