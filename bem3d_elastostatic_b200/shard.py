"""Sharding of the independent parts of the hot path over ranks (one process per GPU).

compute_internal_points (stress_mod.f90:740-776) evaluates every internal point on
its own: the reference loops over points with OpenMP.  Here each rank takes one
contiguous block of points (``shard_range``), evaluates it on its own GPU and the
blocks are all-gathered in rank order, so every rank ends with the same arrays as a
single-GPU run.  The dense solve does not shard (it runs as a replica on each rank).

The gather goes through ``torch.distributed``: NCCL tensors on the rank's GPU, or
CPU tensors with the ``gloo`` backend.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np


def shard_range(count: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous block [p0, p1) of ``count`` items for ``rank`` of ``world``: the
    first ``count % world`` ranks take one item more."""
    if world < 1 or not 0 <= rank < world or count < 0:
        raise ValueError(f"bad shard request: count={count} rank={rank} world={world}")
    base, extra = divmod(count, world)
    p0 = rank * base + min(rank, extra)
    return p0, p0 + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist

    return dist


def gather_columns(parts: Sequence[np.ndarray], count: int, group=None) -> Tuple[np.ndarray, ...]:
    """All-gather per-rank column blocks (last axis = items) into full arrays, in rank
    order.  ``parts`` are this rank's blocks of the arrays; every rank passes the same
    number of arrays with the same leading shapes."""
    import torch

    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    device = torch.device("cpu")
    if dist.get_backend(group) == "nccl":
        device = torch.device("cuda", torch.cuda.current_device())
    ranges = [shard_range(count, r, world) for r in range(world)]
    width = max(p1 - p0 for p0, p1 in ranges)
    out = []
    for a in parts:
        a = np.asarray(a, dtype=np.float64)
        lead = a.shape[:-1]
        if a.shape[-1] != ranges[rank][1] - ranges[rank][0]:
            raise ValueError("a part does not match this rank's block")
        pad = np.zeros(lead + (width,))
        pad[..., : a.shape[-1]] = a
        mine = torch.from_numpy(pad).to(device)
        bufs = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(bufs, mine, group=group)
        full = np.concatenate([b.cpu().numpy()[..., : p1 - p0] for b, (p0, p1) in zip(bufs, ranges)],
                              axis=-1)
        out.append(np.asfortranarray(full) if full.ndim > 1 else full)
    return tuple(out)


def sharded_points(fn: Callable[[int, int], Sequence[np.ndarray]], count: int,
                   group=None) -> Tuple[np.ndarray, ...]:
    """Evaluate ``fn(p0, p1)`` on this rank's block of ``count`` points and gather the
    blocks of every returned array (last axis = points) on all ranks."""
    dist = _dist()
    p0, p1 = shard_range(count, dist.get_rank(group), dist.get_world_size(group))
    return gather_columns(fn(p0, p1), count, group)


def internal_points_sharded(q, points: Optional[np.ndarray] = None, kelvin_consistent: bool = False,
                            group=None):
    """compute_internal_points over all ranks of ``group``: ``q`` is this rank's
    :class:`~bem3d_elastostatic_b200.api.Quadesth` holding the solved system (every
    rank solved the same system).  Returns (u, sigma, prin, vm) for all points on
    every rank, identical to a single-GPU call."""
    m = q.mesh
    if points is None:
        points = np.stack([m.cx, m.cy, m.cz], axis=1)
    points = np.asarray(points, dtype=np.float64)

    def fn(p0: int, p1: int):
        if p1 == p0:
            return (np.zeros((3, 0)), np.zeros((6, 0)), np.zeros((3, 0)), np.zeros(0))
        return q.compute_internal_points(points[p0:p1], kelvin_consistent=kelvin_consistent)

    return sharded_points(fn, points.shape[0], group)
