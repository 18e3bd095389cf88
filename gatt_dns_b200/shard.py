"""Multi-GPU plumbing: independent problems sharded across ranks (one process per GPU).

Nothing on the hot path crosses GPUs: a time step of one flow or one Arnoldi problem stays
on one device.  Ranks split the ensemble (boxes, Arnoldi problems), run their share, and
exchange only small host results (Hessenberg matrices) and the elapsed time for the
max-over-ranks clock.  Works with any torch.distributed backend (NCCL between GPUs, gloo
in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def member_range(total, world, rank):
    """Contiguous slice [lo, hi) of `total` problems owned by `rank` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(value, dist=None, device=None):
    """The largest of every rank's `value` (a time), identical on all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def arnoldi_sharded(runner, v0_all, dist=None, device=None):
    """Run the Arnoldi problems of `v0_all` (list of initial disturbances) across ranks.

    `runner(v0_slice) -> H` runs this rank's problems (e.g. ``lambda v: g.arnoldi(base, v, m,
    nsteps, dt)`` on a context whose nbatch is len(v)) and returns H of shape
    (len(v), m+1, m).  Returns every problem's H, in problem order, on every rank.
    """
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    lo, hi = member_range(len(v0_all), world, rank)
    H = np.asarray(runner(v0_all[lo:hi])) if hi > lo else None
    if world == 1:
        return H
    import torch
    shape = None if H is None else H.shape[1:]
    shapes = [None] * world
    dist.all_gather_object(shapes, shape)
    shape = next(s for s in shapes if s is not None)
    counts = [member_range(len(v0_all), world, r) for r in range(world)]
    width = max(h - l for l, h in counts)
    buf = np.zeros((width,) + tuple(shape))
    if H is not None:
        buf[: hi - lo] = H
    t = torch.from_numpy(buf).to(device) if device is not None else torch.from_numpy(buf)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    return np.concatenate([parts[r].cpu().numpy()[: h - l] for r, (l, h) in enumerate(counts)])
