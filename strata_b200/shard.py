"""Sharding the path over GPUs: row strips with an r-row halo.

Every output cell of a radius-r op depends only on the input rows within r
of it, so a raster splits into horizontal strips that ranks compute
independently: rank i computes output rows [y0, y1) from input rows
[y0 - r, y1 + r) clipped to the raster, run as a raster of its own, and
keeps the rows that are not its own edge ring. Rows a strip's own edge ring
covers are either the whole raster's edge ring (kept, they are NaN and
invalid there too) or rows another rank owns (dropped). No data moves
between ranks while computing: there is no collective on the data path.
The only collective a multi-GPU run needs is the max of the ranks' times.
"""
from __future__ import annotations

from typing import List, Tuple


def strips(height: int, world: int) -> List[Tuple[int, int]]:
    """Output rows [y0, y1) of each rank: contiguous, as equal as can be."""
    if world < 1:
        raise ValueError("world must be at least 1")
    base, extra = divmod(height, world)
    out, y = [], 0
    for i in range(world):
        n = base + (1 if i < extra else 0)
        out.append((y, y + n))
        y += n
    return out


def halo_rows(height: int, radius: int, y0: int, y1: int) -> Tuple[int, int]:
    """Input rows [s0, s1) a strip of output rows [y0, y1) reads."""
    return max(0, y0 - radius), min(height, y1 + radius)


def kept_rows(height: int, radius: int, y0: int, y1: int) -> Tuple[int, int]:
    """Rows of the strip's own result, relative to its first input row,
    that are rank-owned output rows [y0, y1): (k0, k1)."""
    s0, _ = halo_rows(height, radius, y0, y1)
    return y0 - s0, y1 - s0


def assign_rasters(cells: List[int], world: int) -> List[List[int]]:
    """Whole rasters to ranks, greedily by cell count (largest first onto
    the least loaded rank): the split for many independent rasters."""
    loads = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(cells)), key=lambda i: -cells[i]):
        r = min(range(world), key=lambda k: loads[k])
        out[r].append(i)
        loads[r] += cells[i]
    for o in out:
        o.sort()
    return out


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over the ranks of the default process group (or
    the value itself outside one): how a multi-GPU step time is taken."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
