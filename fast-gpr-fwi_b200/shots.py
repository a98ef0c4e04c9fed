"""Shots across ranks: one process per GPU, each solving its own shots.

The reference solves all shots of an epoch on one GPU (src/compute.py:33-50,
`step` shots in one batch).  The path has no exchange between shots inside a
solve, so a multi-GPU run gives each rank a contiguous range of shots and
exchanges data once per gradient: the unnormalised imaging sums of every rank
are added up, then the L2 normalisation of the reference's Backward
(src/compute.py:1174-1180) is applied to the total.  Traces need no exchange
(each rank returns the traces of its own shots).
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch


def shot_range(shots: int, rank: int, world: int) -> Tuple[int, int]:
    """First shot and shot count of `rank` when `shots` shots are split over
    `world` ranks: contiguous ranges, sizes differing by at most one, lower
    ranks taking the larger ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    if shots < 0:
        raise ValueError("negative shot count")
    base, extra = divmod(shots, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def combine_gradients(ge: Optional[torch.Tensor], gs: Optional[torch.Tensor], normalize: bool = True,
                      group=None) -> None:
    """Sum the unnormalised imaging sums (g_eps, g_sigma) of all ranks in place
    and, with `normalize`, divide each by the L2 norm of its total.

    The sums are added and normed in float64 (the accumulators of one solve
    are float64 too) and rounded to float32 once, so every rank ends with the
    same bits.  A rank's tensors must come from adjoint_reference(...,
    normalize=False).  Every rank makes the same collective calls in the same
    order (one all-reduce per tensor present)."""
    for g in (ge, gs):
        if g is None:
            continue
        t = g.to(torch.float64)
        if torch.distributed.is_initialized() and torch.distributed.get_world_size(group) > 1:
            torch.distributed.all_reduce(t, group=group)
        if normalize:
            t = t / torch.linalg.vector_norm(t)
        g.copy_(t)
