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


def allreduce_grads(grads: Dict[str, object], dist) -> None:
    """Sum every gradient table over the ranks, in place, in a fixed order
    (every rank issues the same collectives in the same order)."""
    for name in GRAD_TABLES:
        if name in grads and grads[name] is not None:
            dist.all_reduce(grads[name])


def max_over_ranks(values: List[float], dist, device) -> List[float]:
    """Element-wise max of per-rank timings (device-measured milliseconds)."""
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]
