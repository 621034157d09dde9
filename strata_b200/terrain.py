"""terrain: Horn gradient, slope, aspect and hillshade, Zevenbergen-Thorne
curvature and ruggedness on the device backend, with the reference's entry
points (terrain/gradient.go, slope.go, aspect.go, hillshade.go,
curvature.go, ruggedness.go): the plain function, its Tiled form (with a
Context and engine Options) and its Chunked form (sources and sinks).

Option resolution and its checks run in libstrata_cuda's stage builders
(strata_stage_*), which follow the reference's option code; a programming
error raises StrataPanic with the reference's message.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _lib
from .engine import Background, Context, Options, StageList, process, process_chunked
from .raster import Float32Raster

SlopeDegrees, SlopePercent, SlopeRadians = 0, 1, 2
CurvatureProfile, CurvaturePlan, CurvatureMean = 0, 1, 2
RuggednessTRI, RuggednessTRIWilson, RuggednessTPI, RuggednessRoughness = 0, 1, 2, 3
AspectFlat = -1
MaxRadius = 8


@dataclass
class GradientOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0


@dataclass
class SlopeOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    Units: int = SlopeDegrees


@dataclass
class AspectOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    ZeroForFlat: bool = False
    Trigonometric: bool = False


@dataclass
class HillshadeOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    Azimuth: float = 0.0
    Altitude: float = 0.0


@dataclass
class CurvatureOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    Type: int = CurvatureProfile


# terrain.HeatLoadEquation and terrain.OrientationComponent.
HeatLoadEquation1, HeatLoadEquation2, HeatLoadEquation3 = 0, 1, 2
Northness, Eastness = 0, 1


@dataclass
class HeatLoadOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    Latitude: float = 0.0
    Equation: int = HeatLoadEquation1
    Radiation: bool = False
    Linear: bool = False


@dataclass
class OrientationOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    Component: int = Northness
    Unweighted: bool = False


@dataclass
class RuggednessOptions:
    Type: int = RuggednessTRI
    Radius: int = 0


def _one(fn, copts) -> StageList:
    st = _lib.Stage()
    _lib.check(fn(ctypes.byref(copts), ctypes.byref(st)))
    return StageList().add(st)


def gradient_stage(o: GradientOptions) -> StageList:
    return _one(_lib.lib().strata_stage_gradient,
                _lib.GradientOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, 0))


def slope_stage(o: SlopeOptions) -> StageList:
    return _one(_lib.lib().strata_stage_slope,
                _lib.SlopeOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, o.Units))


def aspect_stage(o: AspectOptions) -> StageList:
    return _one(_lib.lib().strata_stage_aspect,
                _lib.AspectOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, int(bool(o.ZeroForFlat)),
                                   int(bool(o.Trigonometric)), 0))


def hillshade_stage(o: HillshadeOptions) -> StageList:
    return _one(_lib.lib().strata_stage_hillshade,
                _lib.HillshadeOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, 0, o.Azimuth, o.Altitude))


def curvature_stage(o: CurvatureOptions) -> StageList:
    return _one(_lib.lib().strata_stage_curvature,
                _lib.CurvatureOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, o.Type))


def heatload_stage(o: HeatLoadOptions) -> StageList:
    """terrain.heatLoadOp (terrain/heatload.go:144-151). The stage points at
    the regression's terms the builder writes into its options, which the
    StageList keeps."""
    copts = _lib.HeatLoadOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, o.Equation, o.Latitude,
                                 int(bool(o.Radiation)), int(bool(o.Linear)))
    st = _lib.Stage()
    _lib.check(_lib.lib().strata_stage_heatload(ctypes.byref(copts), ctypes.byref(st)))
    return StageList().add(st, copts)


def orientation_stage(o: OrientationOptions) -> StageList:
    return _one(_lib.lib().strata_stage_orientation,
                _lib.OrientationOptions(o.CellSize, o.CellSizeY, o.ZFactor, o.FitRadius, o.Component,
                                        int(bool(o.Unweighted)), 0))


def ruggedness_stage(o: RuggednessOptions) -> StageList:
    return _one(_lib.lib().strata_stage_ruggedness, _lib.RuggednessOptions(o.Type, o.Radius))


def _plain(stages, dem, *outs):
    process(stages, list(outs), [dem], Options(Workers=1), Background())


# Features (terrain/features.go): several ops over one DEM in one call.
@dataclass
class Feature:
    Op: object  # SlopeOptions, AspectOptions, HillshadeOptions, HeatLoadOptions, OrientationOptions,
    # CurvatureOptions or RuggednessOptions
    Dst: Float32Raster


_FEATURE_STAGES = {
    SlopeOptions: slope_stage,
    AspectOptions: aspect_stage,
    HillshadeOptions: hillshade_stage,
    HeatLoadOptions: heatload_stage,
    OrientationOptions: orientation_stage,
    CurvatureOptions: curvature_stage,
    RuggednessOptions: ruggedness_stage,
}


def _feature_stage(i: int, op) -> StageList:
    from .raster import StrataPanic

    if op is None:
        raise StrataPanic(f"terrain: Features output {i} has no Op")
    fn = _FEATURE_STAGES.get(type(op))
    if fn is None:
        raise StrataPanic(f"terrain: Features output {i}: {type(op).__name__} is not a feature op")
    return fn(op)


def Features(out, dem: Float32Raster) -> None:
    FeaturesTiled(Background(), out, dem, Options(Workers=1))


def FeaturesTiled(ctx: Context, out, dem: Float32Raster, eopts: Options):
    from .engine import process_features
    from .raster import StrataPanic

    if not out:
        raise StrataPanic("terrain: Features has no outputs")
    return process_features([_feature_stage(i, f.Op) for i, f in enumerate(out)], [f.Dst for f in out], dem,
                            eopts, ctx)


# Surface (terrain/surface.go): the Horn gradient and the products that
# finish it, from one DEM pass.
@dataclass
class SurfaceOptions:
    CellSize: float = 0.0
    CellSizeY: float = 0.0
    ZFactor: float = 0.0
    FitRadius: int = 0
    Units: int = SlopeDegrees
    ZeroForFlat: bool = False
    Trigonometric: bool = False
    Azimuth: float = 0.0
    Altitude: float = 0.0


@dataclass
class SurfaceOutputs:
    Dx: Float32Raster = None
    Dy: Float32Raster = None
    Slope: Float32Raster = None
    Aspect: Float32Raster = None
    Hillshade: Float32Raster = None


def Surface(out: SurfaceOutputs, dem: Float32Raster, opts: SurfaceOptions) -> None:
    SurfaceTiled(Background(), out, dem, opts, Options(Workers=1))


def SurfaceTiled(ctx: Context, out: SurfaceOutputs, dem: Float32Raster, opts: SurfaceOptions, eopts: Options):
    from .engine import process_features
    from .raster import NewFloat32Like, StrataPanic

    c = dict(CellSize=opts.CellSize, CellSizeY=opts.CellSizeY, ZFactor=opts.ZFactor, FitRadius=opts.FitRadius)
    features, dsts = [], []
    if out.Dx is not None or out.Dy is not None:
        features.append(gradient_stage(GradientOptions(**c)))
        like = out.Dx if out.Dx is not None else out.Dy
        dsts += [out.Dx if out.Dx is not None else NewFloat32Like(like),
                 out.Dy if out.Dy is not None else NewFloat32Like(like)]
    if out.Slope is not None:
        features.append(slope_stage(SlopeOptions(Units=opts.Units, **c)))
        dsts.append(out.Slope)
    if out.Aspect is not None:
        features.append(aspect_stage(AspectOptions(ZeroForFlat=opts.ZeroForFlat, Trigonometric=opts.Trigonometric,
                                                   **c)))
        dsts.append(out.Aspect)
    if out.Hillshade is not None:
        features.append(hillshade_stage(HillshadeOptions(Azimuth=opts.Azimuth, Altitude=opts.Altitude, **c)))
        dsts.append(out.Hillshade)
    if not features:
        raise StrataPanic("terrain: Surface has no outputs; set at least one of Dx, Dy, Slope, Aspect and Hillshade")
    return process_features(features, dsts, dem, eopts, ctx)


# Gradient (terrain/gradient.go)
def Gradient(dx: Float32Raster, dy: Float32Raster, dem: Float32Raster, opts: GradientOptions) -> None:
    _plain(gradient_stage(opts), dem, dx, dy)


def GradientTiled(ctx: Context, dx, dy, dem, opts: GradientOptions, eopts: Options):
    return process(gradient_stage(opts), [dx, dy], [dem], eopts, ctx)


def GradientChunked(ctx: Context, dx, dy, dem, opts: GradientOptions, eopts: Options):
    return process_chunked(gradient_stage(opts), [dx, dy], [dem], eopts, ctx)


# Slope (terrain/slope.go)
def Slope(dst: Float32Raster, dem: Float32Raster, opts: SlopeOptions) -> None:
    _plain(slope_stage(opts), dem, dst)


def SlopeTiled(ctx: Context, dst, dem, opts: SlopeOptions, eopts: Options):
    return process(slope_stage(opts), [dst], [dem], eopts, ctx)


def SlopeChunked(ctx: Context, dst, dem, opts: SlopeOptions, eopts: Options):
    return process_chunked(slope_stage(opts), [dst], [dem], eopts, ctx)


# Aspect (terrain/aspect.go)
def Aspect(dst: Float32Raster, dem: Float32Raster, opts: AspectOptions) -> None:
    _plain(aspect_stage(opts), dem, dst)


def AspectTiled(ctx: Context, dst, dem, opts: AspectOptions, eopts: Options):
    return process(aspect_stage(opts), [dst], [dem], eopts, ctx)


def AspectChunked(ctx: Context, dst, dem, opts: AspectOptions, eopts: Options):
    return process_chunked(aspect_stage(opts), [dst], [dem], eopts, ctx)


# Hillshade (terrain/hillshade.go)
def Hillshade(dst: Float32Raster, dem: Float32Raster, opts: HillshadeOptions) -> None:
    _plain(hillshade_stage(opts), dem, dst)


def HillshadeTiled(ctx: Context, dst, dem, opts: HillshadeOptions, eopts: Options):
    return process(hillshade_stage(opts), [dst], [dem], eopts, ctx)


def HillshadeChunked(ctx: Context, dst, dem, opts: HillshadeOptions, eopts: Options):
    return process_chunked(hillshade_stage(opts), [dst], [dem], eopts, ctx)


# Curvature (terrain/curvature.go)
def Curvature(dst: Float32Raster, dem: Float32Raster, opts: CurvatureOptions) -> None:
    _plain(curvature_stage(opts), dem, dst)


def CurvatureTiled(ctx: Context, dst, dem, opts: CurvatureOptions, eopts: Options):
    return process(curvature_stage(opts), [dst], [dem], eopts, ctx)


def CurvatureChunked(ctx: Context, dst, dem, opts: CurvatureOptions, eopts: Options):
    return process_chunked(curvature_stage(opts), [dst], [dem], eopts, ctx)


# Ruggedness (terrain/ruggedness.go)
def Ruggedness(dst: Float32Raster, dem: Float32Raster, opts: RuggednessOptions) -> None:
    _plain(ruggedness_stage(opts), dem, dst)


def RuggednessTiled(ctx: Context, dst, dem, opts: RuggednessOptions, eopts: Options):
    return process(ruggedness_stage(opts), [dst], [dem], eopts, ctx)


def RuggednessChunked(ctx: Context, dst, dem, opts: RuggednessOptions, eopts: Options):
    return process_chunked(ruggedness_stage(opts), [dst], [dem], eopts, ctx)


def HeatLoad(dst: Float32Raster, dem: Float32Raster, opts: HeatLoadOptions) -> None:
    _plain(heatload_stage(opts), dem, dst)


def HeatLoadTiled(ctx: Context, dst, dem, opts: HeatLoadOptions, eopts: Options):
    return process(heatload_stage(opts), [dst], [dem], eopts, ctx)


def HeatLoadChunked(ctx: Context, dst, dem, opts: HeatLoadOptions, eopts: Options):
    return process_chunked(heatload_stage(opts), [dst], [dem], eopts, ctx)


def Orientation(dst: Float32Raster, dem: Float32Raster, opts: OrientationOptions) -> None:
    _plain(orientation_stage(opts), dem, dst)


def OrientationTiled(ctx: Context, dst, dem, opts: OrientationOptions, eopts: Options):
    return process(orientation_stage(opts), [dst], [dem], eopts, ctx)


def OrientationChunked(ctx: Context, dst, dem, opts: OrientationOptions, eopts: Options):
    return process_chunked(orientation_stage(opts), [dst], [dem], eopts, ctx)
