"""One transfer over several GPUs: target sharding, one process per GPU.

The reference runs a transfer on one device.  Here every rank builds the same
plan (the patch cover depends on all sources and all targets), keeps its shard
of the targets (``Plan.shard``: Morton ranges balanced by the patches' solve
cost), solves only the patches those targets need, and writes their values,
bit-identical to the one-GPU transfer, with zeros at the other targets.  One
all-reduce (sum) over the ranks then assembles the whole result exactly: every
target is owned by exactly one rank and x + 0 = x.  Outputs can also stay
sharded (``gather=False``), with no collective at all.
"""
from __future__ import annotations

import numpy as np

from . import rbf as _rbf


def assemble(out, group=None):
    """Sum of the ranks' sharded outputs, in place (numpy arrays or torch
    tensors; host data goes through the device for an NCCL group)."""
    import torch
    import torch.distributed as dist
    if isinstance(out, np.ndarray):
        t = torch.from_numpy(out)
        if dist.get_backend(group) == "nccl":
            d = t.to(torch.device("cuda", torch.cuda.current_device()))
            dist.all_reduce(d, op=dist.ReduceOp.SUM, group=group)
            t.copy_(d.cpu())
        else:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return out
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out


def interpolate_sharded(space_dimension, rbf_function, source_points, source_values,
                        target_points, *, group=None, gather=True, nodes_per_cluster=50,
                        relative_overlap=0.15, support_radius=0.1, precision="fp64",
                        stats=None):
    """``pacman.rbf.interpolate`` split over the ranks of ``group`` (every
    rank passes the same arguments; each uses its current CUDA device).
    Returns the whole result on every rank (``gather=True``) or this rank's
    shard (its targets' values, zeros elsewhere), and the owned target
    indices are ``Plan.owned_targets()`` of the same cut."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    plan = _rbf.Plan(space_dimension, source_points, target_points,
                     nodes_per_cluster=nodes_per_cluster, relative_overlap=relative_overlap,
                     support_radius=support_radius, precision=precision)
    try:
        if world > 1:
            plan.shard(rank, world)
        out = plan.execute(rbf_function, source_values, stats=stats)
    finally:
        plan.close()
    if gather and world > 1:
        assemble(out, group)
    return out
