"""transfer: Lookup, Reclass and Rescale (transfer/transfer.go:21-92, tiled.go) on
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


def rescale_stage(a: float, b: float) -> StageList:
    """rescaleKernel's chain step (transfer/tiled.go:108-110): vec.OpAffine,
    float32(v*a) + b with no FMA."""
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_rescale(a, b, ctypes.byref(st)))
    return StageList().add(st)


def rescale_range_stage(in_lo: float, in_hi: float, out_lo: float, out_hi: float) -> StageList:
    """RescaleRange's coefficients (transfer/transfer.go:236-250), checked,
    as the Affine step."""
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_rescale_range(in_lo, in_hi, out_lo, out_hi, ctypes.byref(st)))
    return StageList().add(st)


def Rescale(dst: Float32Raster, src: Float32Raster, a: float, b: float) -> None:
    """transfer.Rescale: float32(v*a) + b cell by cell."""
    process(rescale_stage(a, b), [dst], [src], Options(Workers=1))


def RescaleTiled(ctx: Context, dst, src, a, b, eopts: Options):
    return process(rescale_stage(a, b), [dst], [src], eopts, ctx)


def RescaleChunked(ctx: Context, dst, src, a, b, eopts: Options):
    return process_chunked(rescale_stage(a, b), [dst], [src], eopts, ctx)


def RescaleRange(dst: Float32Raster, src: Float32Raster, in_lo, in_hi, out_lo, out_hi) -> None:
    """transfer.RescaleRange: the affine map sending [in_lo, in_hi] to
    [out_lo, out_hi] (no clamp)."""
    process(rescale_range_stage(in_lo, in_hi, out_lo, out_hi), [dst], [src], Options(Workers=1))


def RescaleRangeTiled(ctx: Context, dst, src, in_lo, in_hi, out_lo, out_hi, eopts: Options):
    return process(rescale_range_stage(in_lo, in_hi, out_lo, out_hi), [dst], [src], eopts, ctx)


def RescaleRangeChunked(ctx: Context, dst, src, in_lo, in_hi, out_lo, out_hi, eopts: Options):
    return process_chunked(rescale_range_stage(in_lo, in_hi, out_lo, out_hi), [dst], [src], eopts, ctx)
