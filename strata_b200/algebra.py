"""algebra: the cell-by-cell raster operations (algebra/algebra.go,
tiled.go) on the device backend, each one vec.Chain step run by the
pointwise kernel.

The binary operations (Add, Sub, Mul, Min, Max) read two rasters of one
size; the output is valid where every masked input is (pointwise.
BinaryValidity). Clamp is one step over one input. Mask copies src where
src and mask are both valid: on the device that is the chain max(v, v)
over (src, mask), which is v for every cell (a NaN stays a NaN, -0 stays
-0), with the validity the AND of both inputs'.
"""
from __future__ import annotations

from .engine import Context, Options, StageList, process, process_chunked
from .raster import Float32Raster, NotSupported
from .vec import OpAdd, OpClamp, OpMax, OpMin, OpMul, OpSub, step_stage


def binary_stage(op: int) -> StageList:
    """The chain step of a binary operation: acc op input 1."""
    return step_stage(op, 1)


def clamp_stage(lo: float, hi: float) -> StageList:
    """clampKernel's chain step (algebra/tiled.go:122-124): min(max(v, lo), hi)."""
    return step_stage(OpClamp, -1, lo, hi)


def _binary(op: int, dst: Float32Raster, a: Float32Raster, b: Float32Raster, eopts=None, ctx=None):
    return process(binary_stage(op), [dst], [a, b], eopts or Options(Workers=1), ctx)


def Add(dst, a, b) -> None:
    """algebra.Add: dst = a + b."""
    _binary(OpAdd, dst, a, b)


def Sub(dst, a, b) -> None:
    """algebra.Sub: dst = a - b."""
    _binary(OpSub, dst, a, b)


def Mul(dst, a, b) -> None:
    """algebra.Mul: dst = a * b."""
    _binary(OpMul, dst, a, b)


def Min(dst, a, b) -> None:
    """algebra.Min: Go's min (NaN wins, -0 below +0)."""
    _binary(OpMin, dst, a, b)


def Max(dst, a, b) -> None:
    """algebra.Max: Go's max (NaN wins, +0 above -0)."""
    _binary(OpMax, dst, a, b)


def AddTiled(ctx: Context, dst, a, b, eopts: Options):
    return _binary(OpAdd, dst, a, b, eopts, ctx)


def SubTiled(ctx: Context, dst, a, b, eopts: Options):
    return _binary(OpSub, dst, a, b, eopts, ctx)


def MulTiled(ctx: Context, dst, a, b, eopts: Options):
    return _binary(OpMul, dst, a, b, eopts, ctx)


def MinTiled(ctx: Context, dst, a, b, eopts: Options):
    return _binary(OpMin, dst, a, b, eopts, ctx)


def MaxTiled(ctx: Context, dst, a, b, eopts: Options):
    return _binary(OpMax, dst, a, b, eopts, ctx)


def Clamp(dst: Float32Raster, src: Float32Raster, lo: float, hi: float) -> None:
    """algebra.Clamp: min(max(src, lo), hi) cell by cell."""
    process(clamp_stage(lo, hi), [dst], [src], Options(Workers=1))


def ClampTiled(ctx: Context, dst, src, lo, hi, eopts: Options):
    return process(clamp_stage(lo, hi), [dst], [src], eopts, ctx)


def ClampChunked(ctx: Context, dst, src, lo, hi, eopts: Options):
    return process_chunked(clamp_stage(lo, hi), [dst], [src], eopts, ctx)


def Mask(dst: Float32Raster, src: Float32Raster, mask: Float32Raster) -> None:
    """algebra.Mask: src's cells, valid where src and mask both are."""
    process(step_stage(OpMax, 0), [dst], [src, mask], Options(Workers=1))


def MaskTiled(ctx: Context, dst, src, mask, eopts: Options):
    return process(step_stage(OpMax, 0), [dst], [src, mask], eopts, ctx)


def _no_chunked(name: str):
    def f(*args, **kwargs):
        raise NotSupported(f"algebra.{name}Chunked: a chain over two inputs has no chunked form on the gpu backend")
    return f


AddChunked, SubChunked, MulChunked = _no_chunked("Add"), _no_chunked("Sub"), _no_chunked("Mul")
MinChunked, MaxChunked, MaskChunked = _no_chunked("Min"), _no_chunked("Max"), _no_chunked("Mask")
