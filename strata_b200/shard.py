"""Sharding the path over GPUs: row strips with an r-row halo.

Every output cell of a radius-r op depends only on the input rows within r
of it, so a raster splits into horizontal strips that ranks compute
independently: rank i computes output rows [y0, y1) from input rows
[y0 - r, y1 + r) clipped to the raster, run as a raster of its own, and
keeps the rows that are not its own edge ring. Rows a strip's own edge ring
covers are either the whole raster's edge ring (kept, they are NaN and
invalid there too) or rows another rank owns (dropped). No data moves
between ranks while computing: there is no collective on the data path.
The only collective a multi-GPU run needs is the max of the ranks' times,
and, when every rank wants the whole result, the exchange of the strips
(process_sharded). In one process, engine.Options(Devices=[...]) runs the
same split over several GPUs (strata_process_multi).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple


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


def stage_radius(stages) -> int:
    """How far the pipeline's first stage reads (its tail is pointwise): the
    fit's radius, 1 for the Horn and Zevenbergen-Thorne products, 0 for a
    pointwise pipeline, else the stage's radius."""
    from . import _lib

    st = stages.stages[0]
    if st.flags & _lib.STAGE_FIT:
        return int(st.radius)
    if st.op in (_lib.OP_GRADIENT, _lib.OP_SLOPE, _lib.OP_ASPECT, _lib.OP_HILLSHADE, _lib.OP_CURVATURE,
                 _lib.OP_HEATLOAD, _lib.OP_ORIENTATION):
        return 1
    if st.op in (_lib.OP_LOOKUP, _lib.OP_RECLASS, _lib.OP_STEP):
        return 0
    return int(st.radius)


def process_sharded(stages, dst, src, rank: Optional[int] = None, world: Optional[int] = None, opts=None,
                    compute: Optional[Callable] = None, group=None) -> None:
    """One raster over the ranks of a process group, one rank a GPU: every
    rank holds the host input src and outputs dst; rank i computes output
    rows strips(H, world)[i] from their halo rows on its own device
    (engine.process_strip, the same rows strata_process writes), then the
    strips are exchanged so that every rank's dst holds the whole result.
    No data moves between ranks while computing; the exchange is the
    reassembly. compute replaces the device call (same arguments as
    engine.process_strip) where a rank has no GPU."""
    import numpy as np

    from . import engine
    from .raster import Float32Raster, mask_from_bool

    if rank is None or world is None:
        import torch.distributed as dist

        rank, world = dist.get_rank(group), dist.get_world_size(group)
    H, W = src.height, src.width
    r = stage_radius(stages)
    y0, y1 = strips(H, world)[rank]
    if y1 > y0:
        s0, s1 = halo_rows(H, r, y0, y1)
        (compute or engine.process_strip)(stages, [d.Window(0, y0, W, y1 - y0) for d in dst],
                                          src.Window(0, s0, W, s1 - s0), H, s0, y0, opts)
    if world == 1:
        return None
    import torch.distributed as dist

    mine = [(d.Window(0, y0, W, y1 - y0).numpy(), d.Window(0, y0, W, y1 - y0).valid_numpy()) if y1 > y0 else None
            for d in dst]
    got = [None] * world
    dist.all_gather_object(got, (y0, y1, mine), group=group)
    for k, (a0, a1, parts) in enumerate(got):
        if k == rank or a1 <= a0:
            continue
        for d, (cells, valid) in zip(dst, parts):
            win = d.Window(0, a0, W, a1 - a0)
            part = Float32Raster(np.ascontiguousarray(cells).reshape(-1), W, a1 - a0, W,
                                 None if valid is None else mask_from_bool(valid, W, 0), 0)
            engine._copy_cells(win, part, valid is not None and win.valid is not None)
    return None
