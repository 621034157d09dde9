"""focal: weighted, separable and box neighbourhood operations at radius
1-8 on the device backend, with the reference's entry points
(focal/correlate.go, separable.go, box.go): plain, Tiled and Chunked.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _lib
from .engine import Background, Context, Options, StageList, process, process_chunked
from .raster import Float32Raster

MaxRadius = 8


@dataclass
class WeightsOptions:
    Radius: int = 0
    Weights: List[float] = field(default_factory=list)


@dataclass
class SeparableOptions:
    Radius: int = 0
    Row: List[float] = field(default_factory=list)
    Col: List[float] = field(default_factory=list)


@dataclass
class BoxOptions:
    Radius: int = 0


def _f32(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(-1))


def weights_stage(o: WeightsOptions, convolve: bool) -> StageList:
    w = _f32(o.Weights)
    co = _lib.WeightsOptions(o.Radius, w.size, w.ctypes.data if w.size else None)
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_correlate(ctypes.byref(co), 1 if convolve else 0, ctypes.byref(st)))
    return StageList().add(st, w)


def separable_stage(o: SeparableOptions) -> StageList:
    row, col = _f32(o.Row), _f32(o.Col)
    co = _lib.SeparableOptions(o.Radius, row.size, row.ctypes.data if row.size else None, col.size, 0,
                               col.ctypes.data if col.size else None)
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_separable(ctypes.byref(co), ctypes.byref(st)))
    return StageList().add(st, row, col)


def box_stage(o: BoxOptions, op: int) -> StageList:
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_box(ctypes.byref(_lib.BoxOptions(o.Radius)), op, ctypes.byref(st)))
    return StageList().add(st)


def Gaussian(radius: int, sigma: float) -> np.ndarray:
    """focal.Gaussian (focal/separable.go:59-76): 2·radius+1 normalised taps."""
    out = (ctypes.c_float * (2 * max(radius, 0) + 1))()
    _lib.check(_lib.lib().strata_focal_gaussian(radius, sigma, out))
    return np.array(list(out), dtype=np.float32)


def _plain(stages, dst, src):
    process(stages, [dst], [src], Options(Workers=1), Background())


def Correlate(dst: Float32Raster, src: Float32Raster, opts: WeightsOptions) -> None:
    _plain(weights_stage(opts, False), dst, src)


def CorrelateTiled(ctx: Context, dst, src, opts: WeightsOptions, eopts: Options):
    return process(weights_stage(opts, False), [dst], [src], eopts, ctx)


def CorrelateChunked(ctx: Context, dst, src, opts: WeightsOptions, eopts: Options):
    return process_chunked(weights_stage(opts, False), [dst], [src], eopts, ctx)


def Convolve(dst: Float32Raster, src: Float32Raster, opts: WeightsOptions) -> None:
    _plain(weights_stage(opts, True), dst, src)


def ConvolveTiled(ctx: Context, dst, src, opts: WeightsOptions, eopts: Options):
    return process(weights_stage(opts, True), [dst], [src], eopts, ctx)


def ConvolveChunked(ctx: Context, dst, src, opts: WeightsOptions, eopts: Options):
    return process_chunked(weights_stage(opts, True), [dst], [src], eopts, ctx)


def CorrelateSeparable(dst: Float32Raster, src: Float32Raster, opts: SeparableOptions) -> None:
    _plain(separable_stage(opts), dst, src)


def CorrelateSeparableTiled(ctx: Context, dst, src, opts: SeparableOptions, eopts: Options):
    return process(separable_stage(opts), [dst], [src], eopts, ctx)


def CorrelateSeparableChunked(ctx: Context, dst, src, opts: SeparableOptions, eopts: Options):
    return process_chunked(separable_stage(opts), [dst], [src], eopts, ctx)


def Mean(dst: Float32Raster, src: Float32Raster, opts: BoxOptions) -> None:
    _plain(box_stage(opts, _lib.OP_MEAN), dst, src)


def MeanTiled(ctx: Context, dst, src, opts: BoxOptions, eopts: Options):
    return process(box_stage(opts, _lib.OP_MEAN), [dst], [src], eopts, ctx)


def MeanChunked(ctx: Context, dst, src, opts: BoxOptions, eopts: Options):
    return process_chunked(box_stage(opts, _lib.OP_MEAN), [dst], [src], eopts, ctx)


def Min(dst: Float32Raster, src: Float32Raster, opts: BoxOptions) -> None:
    _plain(box_stage(opts, _lib.OP_MIN), dst, src)


def MinTiled(ctx: Context, dst, src, opts: BoxOptions, eopts: Options):
    return process(box_stage(opts, _lib.OP_MIN), [dst], [src], eopts, ctx)


def MinChunked(ctx: Context, dst, src, opts: BoxOptions, eopts: Options):
    return process_chunked(box_stage(opts, _lib.OP_MIN), [dst], [src], eopts, ctx)


def Max(dst: Float32Raster, src: Float32Raster, opts: BoxOptions) -> None:
    _plain(box_stage(opts, _lib.OP_MAX), dst, src)


def MaxTiled(ctx: Context, dst, src, opts: BoxOptions, eopts: Options):
    return process(box_stage(opts, _lib.OP_MAX), [dst], [src], eopts, ctx)


def MaxChunked(ctx: Context, dst, src, opts: BoxOptions, eopts: Options):
    return process_chunked(box_stage(opts, _lib.OP_MAX), [dst], [src], eopts, ctx)
