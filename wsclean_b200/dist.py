"""Visibility-sharded gridding across ranks (one process per GPU).

The w-gridder is linear in the visibilities, so ranks may each grid a
contiguous block of rows and sum their partial images: the sum over ranks is
the path's one exchange step (an all-reduce of the FP64 dirty image; NCCL over
NVLink on GPUs).  Degridding needs no exchange: each rank predicts its own
rows from the replicated model image.  The benchmark runs independent
replicas instead (one full workload per GPU); this module is the sharded
form for a single large job.
"""
from __future__ import annotations


def shard_rows(nrows, rank, world):
    """Contiguous row block [lo, hi) of a rank."""
    lo = (nrows * rank) // world
    hi = (nrows * (rank + 1)) // world
    return lo, hi


def sharded_ms2dirty(grid_fn, uvw, freq, vis, group=None, **kw):
    """grid_fn(uvw, freq, vis, **kw) -> partial dirty image (torch tensor);
    returns the all-reduced image on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    lo, hi = shard_rows(uvw.shape[0], rank, world)
    part = grid_fn(uvw[lo:hi], freq, vis[lo:hi], **kw)
    part = torch.as_tensor(part).to(torch.float64)
    if world > 1:
        dist.all_reduce(part, op=dist.ReduceOp.SUM, group=group)
    return part


def sharded_dirty2ms(degrid_fn, uvw, freq, dirty, group=None, **kw):
    """Each rank predicts its own rows; returns (lo, hi, local visibilities)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    lo, hi = shard_rows(uvw.shape[0], rank, world)
    return lo, hi, degrid_fn(uvw[lo:hi], freq, dirty, **kw)
