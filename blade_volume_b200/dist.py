"""Data-parallel plumbing of the training step across ranks (one process per
GPU, torch.distributed for the exchange).

Rays are independent, so the walk shards by views: each rank renders and
differentiates its own cameras against its own targets (weak scaling), and
the only exchange of a step is one sum all-reduce of the gradient tables
(density [N], SH [N, 3K], positions [N, 3], radii [N]).  Timing is taken on
each rank's device and reduced with a max.  The reference has no multi-GPU
path; nothing here runs a collective inside a kernel.
"""

from __future__ import annotations

import math
from typing import Dict, List

from . import scenes

GRAD_TABLES = ("d_density", "d_sh", "d_pos", "d_radius")


def rank_cameras(views: int, rank: int, radius: float = 3.0, fov_deg: float = 60.0,
                 aspect: float = 1.0, depth: float = 100.0) -> List[scenes.Camera]:
    """The cameras of one rank: `views` Fibonacci-sphere cameras seeded by
    the rank, so ranks render different views of the same scene."""
    return scenes.sphere_cameras(views, radius, 1 + rank, math.radians(fov_deg), aspect, depth)


def allreduce_grads(grads: Dict[str, object], dist, bucket=None):
    """Sum every gradient table over the ranks, in place, with ONE all-reduce.
    Tables from a tracer's new_grads() are views of one flat buffer
    (``grads.flat``), which is reduced directly.  Otherwise the tables are
    packed into one flat bucket in a fixed order (every rank packs the same
    tables the same way), reduced, and unpacked; ``bucket`` may be a
    preallocated flat tensor of at least the tables' total size (it is
    returned, so a caller can keep it across steps)."""
    import torch

    flat = getattr(grads, "flat", None)
    if flat is not None:
        dist.all_reduce(flat)
        return bucket
    tabs = [grads[n] for n in GRAD_TABLES if grads.get(n) is not None]
    if not tabs:
        return bucket
    total = sum(t.numel() for t in tabs)
    if bucket is None or bucket.numel() < total:
        bucket = torch.empty(total, dtype=tabs[0].dtype, device=tabs[0].device)
    flat = bucket[:total]
    off = 0
    for t in tabs:
        flat[off:off + t.numel()].copy_(t.reshape(-1))
        off += t.numel()
    dist.all_reduce(flat)
    off = 0
    for t in tabs:
        t.copy_(flat[off:off + t.numel()].view_as(t))
        off += t.numel()
    return bucket


def max_over_ranks(values: List[float], dist, device) -> List[float]:
    """Element-wise max of per-rank timings (device-measured milliseconds)."""
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]
