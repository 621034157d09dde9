"""transfer: Lookup and Reclass (transfer/transfer.go:21-46, tiled.go) on
the device backend, and the stage builders a pipeline fuses as its
pointwise tail (see graph.py).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .engine import Context, Options, StageList, process, process_chunked
from .raster import Float32Raster


def _f32(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(-1))


def lookup_stage(xs, ys) -> StageList:
    xa, ya = _f32(xs), _f32(ys)
    if xa.size != ya.size:
        from .raster import StrataPanic

        raise StrataPanic(f"transfer.Lookup: xs and ys must have equal length, got {xa.size} and {ya.size}")
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_lookup(xa.ctypes.data, ya.ctypes.data, xa.size, ctypes.byref(st)))
    return StageList().add(st, xa, ya)


def reclass_stage(breaks, values) -> StageList:
    b, v = _f32(breaks), _f32(values)
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_reclass(b.ctypes.data, b.size, v.ctypes.data, v.size, ctypes.byref(st)))
    return StageList().add(st, b, v)


def Lookup(dst: Float32Raster, src: Float32Raster, xs, ys) -> None:
    """transfer.Lookup: the polyline through (xs, ys), clamped at the ends."""
    process(lookup_stage(xs, ys), [dst], [src], Options(Workers=1))


def LookupTiled(ctx: Context, dst, src, xs, ys, eopts: Options):
    return process(lookup_stage(xs, ys), [dst], [src], eopts, ctx)


def LookupChunked(ctx: Context, dst, src, xs, ys, eopts: Options):
    return process_chunked(lookup_stage(xs, ys), [dst], [src], eopts, ctx)


def Reclass(dst: Float32Raster, src: Float32Raster, breaks, values) -> None:
    """transfer.Reclass: values[k] for k = the number of breaks at or below
    the cell; NaN stays NaN."""
    process(reclass_stage(breaks, values), [dst], [src], Options(Workers=1))


def ReclassTiled(ctx: Context, dst, src, breaks, values, eopts: Options):
    return process(reclass_stage(breaks, values), [dst], [src], eopts, ctx)


def ReclassChunked(ctx: Context, dst, src, breaks, values, eopts: Options):
    return process_chunked(reclass_stage(breaks, values), [dst], [src], eopts, ctx)
