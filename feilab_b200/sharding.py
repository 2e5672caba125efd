"""Slice sharding across GPUs: the host-side logic of multi-GPU runs.

Slices (xz-sections) of a tilt series are independent solves, so ranks share
nothing but the geometry: each rank takes its own slices and no data moves
between GPUs.  The only collective is the timing reduction (max over ranks).

* ``sm_split`` is the reference's partition of a slice range over devices in
  proportion to their SM counts (ICONGPU.cu:398-449): every device but the
  last takes floor(sm_d / sum(sm) * total), the last takes the rest.  The
  icon-gpu tool applies the same rule in C++ (icon_cli.cpp).
* ``rank_slices`` gives a benchmark rank its slice indices for ``nsteps``
  batches of ``per_step`` slices: disjoint between ranks (weak scaling),
  wrapping over the ``ny`` slices of the volume.
* ``max_over_ranks`` reduces a time with MAX over the process group.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def sm_split(total: int, sms: Sequence[int]) -> List[Tuple[int, int]]:
    """(start, count) per device for slices 0..total-1."""
    if total < 0:
        raise ValueError("total must be >= 0")
    if not sms:
        raise ValueError("no devices")
    w = [max(1, int(s)) for s in sms]
    tot = float(sum(w))
    out, start = [], 0
    for d, s in enumerate(w):
        share = total - start if d == len(w) - 1 else int(s / tot * total)
        out.append((start, share))
        start += share
    return out


def rank_slices(rank: int, world: int, nsteps: int, per_step: int, ny: int) -> List[int]:
    """Slice indices of one rank: rank r takes nsteps*per_step consecutive
    indices starting at r*nsteps*per_step, modulo ny."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    n = nsteps * per_step
    return [(rank * n + i) % ny for i in range(n)]


def max_over_ranks(x: float, world: int, device=None) -> float:
    """MAX of x over the default process group (x itself when world == 1)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, per_step: int, steps: int, seconds: float) -> float:
    """Whole-job slices/s: every rank's slices over the slowest rank's time."""
    return world * per_step * steps / seconds
