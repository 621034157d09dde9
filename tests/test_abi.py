"""The C ABI without a GPU: libstrata_cuda loads and exports every entry
point include/strata_cuda.h declares, its structs have the header's layout,
its op codes match the oracle's, and the stage builders resolve options to
the reference's constants and reject what the reference panics on, with
its messages."""
from __future__ import annotations

import ctypes
import math
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as orc
from strata_b200 import _lib, focal, terrain, transfer, vec
from strata_b200.raster import NotSupported, StrataPanic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "strata_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(strata_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    L = _lib.lib()
    for n in names:
        assert hasattr(L, n), f"libstrata_cuda.so does not export {n}"
    # and the binding covers each one
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_abi_version():
    assert _lib.lib().strata_abi_version() == 2


def test_op_codes_match_oracle_and_header():
    text = open(HEADER).read()
    for name, val in re.findall(r"STRATA_OP_(\w+) = (\d+)", text):
        assert getattr(orc, name) == int(val), name
        assert getattr(_lib, "OP_" + name) == int(val), name


def test_struct_layouts_match_header(tmp_path):
    """Compiles a C program against the header and compares sizeof and
    offsetof with the ctypes mirrors."""
    structs = {
        "strata_raster": _lib.Raster, "strata_stage": _lib.Stage, "strata_exec_opts": _lib.ExecOpts,
        "strata_stats": _lib.Stats, "strata_source": _lib.Source, "strata_sink": _lib.Sink,
        "strata_slope_options": _lib.SlopeOptions, "strata_aspect_options": _lib.AspectOptions,
        "strata_hillshade_options": _lib.HillshadeOptions, "strata_curvature_options": _lib.CurvatureOptions,
        "strata_gradient_options": _lib.GradientOptions, "strata_ruggedness_options": _lib.RuggednessOptions,
        "strata_weights_options": _lib.WeightsOptions, "strata_separable_options": _lib.SeparableOptions,
        "strata_box_options": _lib.BoxOptions, "strata_heatload_options": _lib.HeatLoadOptions,
        "strata_orientation_options": _lib.OrientationOptions, "strata_raw_file": _lib.RawFile,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, ct in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split(" ") for line in out if line)
    for cname, ct in structs.items():
        assert int(got[cname]) == ctypes.sizeof(ct), cname
        for fname, _ in ct._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(ct, fname).offset, f"{cname}.{fname}"


# ---------------------------------------------------------------------------
# Stage builders: the reference's option resolution.

def k_of(sl):
    return [np.float32(v) for v in sl.stages[0].k]


@pytest.mark.parametrize("cs,csy,z", [(30, 0, 0), (5, 0, 1), (10, 12.5, -2), (0.25, 0.5, 3.5), (1e-3, 7, 0)])
def test_horn_scales(cs, csy, z):
    st = terrain.slope_stage(terrain.SlopeOptions(CellSize=cs, CellSizeY=csy, ZFactor=z))
    kx, ky = orc.horn_scales(cs, csy or cs, z or 1.0)
    got = k_of(st)
    assert got[0] == kx and got[1] == ky
    assert got[2] == np.float32(180 / math.pi) and st.stages[0].kind == 1


def test_slope_units():
    for units, scale, atan in ((terrain.SlopeDegrees, np.float32(180 / math.pi), 1),
                               (terrain.SlopePercent, np.float32(100), 0), (terrain.SlopeRadians, np.float32(1), 1)):
        st = terrain.slope_stage(terrain.SlopeOptions(CellSize=1, Units=units))
        assert k_of(st)[2] == scale and st.stages[0].kind == atan


@pytest.mark.parametrize("az,alt", [(0, 0), (315, 45), (90, 0), (-45, 30), (725, 89.5), (180, 90)])
def test_hillshade_light(az, alt):
    st = terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=1, Azimuth=az, Altitude=alt))
    assert k_of(st)[2:5] == orc.hillshade_light(az, alt)


def test_aspect_flat_and_trig():
    st = terrain.aspect_stage(terrain.AspectOptions(CellSize=1))
    assert k_of(st)[2] == -1 and st.stages[0].kind == 0
    st = terrain.aspect_stage(terrain.AspectOptions(CellSize=1, ZeroForFlat=True, Trigonometric=True))
    assert k_of(st)[2] == 0 and st.stages[0].kind == 1


@pytest.mark.parametrize("cs,csy,z", [(1, 0, 0), (3, 0.5, -2), (30, 0, 1), (2, 4, 1)])
def test_zt_scales(cs, csy, z):
    st = terrain.curvature_stage(terrain.CurvatureOptions(CellSize=cs, CellSizeY=csy, ZFactor=z, Type=2))
    assert k_of(st)[:5] == orc.zt_scales(cs, csy or cs, z or 1.0)
    assert st.stages[0].kind == 2


@pytest.mark.parametrize("r,sigma", [(1, 0.5), (3, 1.0), (8, 2.5), (5, 10.0)])
def test_gaussian_taps(r, sigma):
    assert (focal.Gaussian(r, sigma).view(np.uint32) == orc.gaussian(r, sigma).view(np.uint32)).all()


def test_ruggedness_radius_default():
    st = terrain.ruggedness_stage(terrain.RuggednessOptions(Type=terrain.RuggednessTPI))
    assert st.stages[0].radius == 1 and st.stages[0].kind == 2


@pytest.mark.parametrize("make,msg", [
    (lambda: terrain.slope_stage(terrain.SlopeOptions()), "terrain: CellSize must be positive and finite, got 0"),
    (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=float("inf"))),
     "terrain: CellSize must be positive and finite, got +Inf"),
    (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=1, CellSizeY=-2)),
     "terrain: CellSizeY must be positive and finite (or 0 for CellSize), got -2"),
    (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=1, ZFactor=float("nan"))),
     "terrain: ZFactor must be finite, got NaN"),
    (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=1, Units=7)), "terrain: unknown SlopeUnits 7"),
    (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=1e-300)),
     "terrain: ZFactor/(8·CellSize) and ZFactor/(8·CellSizeY) must be finite and non-zero as float32, got +Inf"),
    (lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=1, Altitude=91)),
     "terrain: Altitude must be in (0, 90] (or 0 for 45), got 91"),
    (lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=1, Azimuth=float("inf"))),
     "terrain: Azimuth must be finite, got +Inf"),
    (lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=1, Type=3)),
     "terrain: unknown CurvatureType 3"),
    (lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Radius=9)),
     "terrain: RuggednessOptions.Radius must be 0 to 8, got 9"),
    (lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=4)), "terrain: unknown RuggednessType 4"),
    (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=1, FitRadius=9)),
     "terrain: FitRadius must be 0 to 8, got 9"),
    (lambda: focal.weights_stage(focal.WeightsOptions(Radius=0, Weights=[1]), False),
     "focal: Radius must be 1 to 8, got 0"),
    (lambda: focal.weights_stage(focal.WeightsOptions(Radius=1, Weights=[1] * 8), False),
     "focal: Radius 1 needs 3×3 = 9 Weights, got 8"),
    (lambda: focal.weights_stage(focal.WeightsOptions(Radius=1, Weights=[1] * 8 + [float("nan")]), False),
     "focal: Weights must be finite, got NaN at index 8"),
    (lambda: focal.separable_stage(focal.SeparableOptions(Radius=2, Row=[1] * 5, Col=[1] * 4)),
     "focal: Radius 2 needs 5 Row and 5 Col taps, got 5 and 4"),
    (lambda: focal.Gaussian(2, 0), "focal: Gaussian sigma must be positive and finite, got 0"),
    (lambda: transfer.lookup_stage([], []), "transfer.Lookup: the table needs at least one knot"),
    (lambda: transfer.lookup_stage([0, 0], [1, 2]),
     "transfer.Lookup: xs must be strictly increasing, but xs[1] = 0 is not above xs[0] = 0"),
    (lambda: transfer.lookup_stage([0, float("inf")], [1, 2]), "transfer.Lookup: xs must be finite, but xs[1] = +Inf"),
    (lambda: transfer.reclass_stage([1, 2], [1, 2]),
     "transfer.Reclass: values must hold one more element than breaks, got 2 values and 2 breaks"),
    (lambda: transfer.reclass_stage([1, float("nan")], [1, 2, 3]),
     "transfer.Reclass: breaks must not hold NaN, but breaks[1] is NaN"),
    (lambda: transfer.rescale_range_stage(1, 1, 0, 1),
     "transfer.RescaleRange: inLo and inHi must be finite and different, got 1 and 1"),
    (lambda: transfer.rescale_range_stage(0, 1, float("inf"), 1),
     "transfer.RescaleRange: outLo and outHi must be finite, got +Inf and 1"),
    (lambda: transfer.rescale_range_stage(0, 1e-30, -3e38, 3e38),
     "transfer.RescaleRange: [0, 1e-30] to [-3e+38, 3e+38] gives a scale of +Inf"),
    (lambda: vec.step_stage(13), "vec: chain step has unknown operation Op(13)"),
    (lambda: vec.step_stage(vec.OpMin, -1), "vec: chain step (Min) reads input -1, which is not one of its 4"),
    (lambda: vec.step_stage(vec.OpClamp, 1, 0, 1), "vec: chain step (Clamp) reads no input, so its Src must be -1, not 1"),
])
def test_builders_panic_like_the_reference(make, msg):
    with pytest.raises(StrataPanic) as e:
        make()
    assert str(e.value).startswith(msg), str(e.value)


def _k(stages, n):
    return [np.float32(stages.stages[0].k[i]) for i in range(n)]


@pytest.mark.parametrize("r", [1, 2, 5, 8])
def test_fit_stages_resolve_as_the_oracle(r):
    """FitRadius 1..8 builds Wood's fit (terrain/fit.go:38-66): the factors
    the oracle derives, the fit flag and radius, the product's constants
    after them."""
    from oracle import oracle as orc

    want = orc.fit_scales(r, 3.0, 5.0, 2.0)
    g = terrain.gradient_stage(terrain.GradientOptions(CellSize=3, CellSizeY=5, ZFactor=2, FitRadius=r))
    st = g.stages[0]
    assert st.flags == _lib.STAGE_FIT and st.radius == r and _k(g, 5) == want
    sl = terrain.slope_stage(terrain.SlopeOptions(CellSize=3, CellSizeY=5, ZFactor=2, FitRadius=r))
    assert _k(sl, 6) == want + [np.float32(180 / np.pi)] and sl.stages[0].kind == 1
    hs = terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=3, CellSizeY=5, ZFactor=2, FitRadius=r))
    assert _k(hs, 8)[5:] == [np.float32(v) for v in orc.hillshade_light(315, 45)]
    cv = terrain.curvature_stage(terrain.CurvatureOptions(CellSize=3, CellSizeY=5, ZFactor=2, FitRadius=r, Type=2))
    assert cv.stages[0].kind == 2 and _k(cv, 5) == want
    with pytest.raises(StrataPanic, match="FitRadius must be 0 to 8, got 9"):
        terrain.slope_stage(terrain.SlopeOptions(CellSize=1, FitRadius=9))


@pytest.mark.parametrize("lat,eq,rad,lin", [(40.0, 0, False, False), (-33.5, 1, True, True), (60.0, 2, False, True),
                                            (0.0, 0, True, False)])
def test_heatload_stage_terms_as_the_oracle(lat, eq, rad, lin):
    """heatLoadTerms (terrain/heatload.go:110-142): the eight float64 terms
    the stage carries are the oracle's, and Linear takes exp but for
    Equation 3."""
    from oracle import oracle as orc

    st = terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=10, Latitude=lat, Equation=eq, Radiation=rad,
                                                        Linear=lin))
    s0 = st.stages[0]
    assert s0.op == _lib.OP_HEATLOAD and s0.table_len[0] == 16
    got = np.ctypeslib.as_array((ctypes.c_double * 8).from_address(s0.table[0]))
    want, ex = orc.heatload_terms(lat, eq, rad, lin)
    assert np.array_equal(got, want) and s0.kind == int(ex)
    with pytest.raises(StrataPanic, match=r"Latitude must be in \[-90, 90\], got 91"):
        terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=1, Latitude=91))
    with pytest.raises(StrataPanic, match="unknown HeatLoadEquation 3"):
        terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=1, Equation=3))


def test_orientation_stage_kind():
    st = terrain.orientation_stage(terrain.OrientationOptions(CellSize=2, Component=terrain.Eastness,
                                                              Unweighted=True))
    assert st.stages[0].op == _lib.OP_ORIENTATION and st.stages[0].kind == 3
    with pytest.raises(StrataPanic, match="unknown OrientationComponent 2"):
        terrain.orientation_stage(terrain.OrientationOptions(CellSize=1, Component=2))


def test_context_without_a_device_fails_cleanly():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    p = ctypes.c_void_p()
    rc = _lib.lib().strata_ctx_create(0, ctypes.byref(p))
    assert rc in (_lib.ECUDA, _lib.EINVAL)
    assert _lib.last_error()


@pytest.mark.parametrize("lo,hi,olo,ohi", [(0, 10, 100, 200), (-3, 7, 10, 0), (0.1, 0.7, -1, 1), (1e-3, 2e5, 0, 255)])
def test_rescale_range_coefficients_as_the_oracle(lo, hi, olo, ohi):
    st = transfer.rescale_range_stage(lo, hi, olo, ohi).stages[0]
    a, b = orc.rescale_range_coeffs(lo, hi, olo, ohi)
    assert st.op == _lib.OP_STEP and st.kind == vec.OpAffine and st.input == -1
    assert np.float32(st.k[0]) == a and np.float32(st.k[1]) == b


def test_step_stage_fields():
    st = vec.step_stage(vec.OpSub, 3).stages[0]
    assert (st.op, st.kind, st.input) == (_lib.OP_STEP, vec.OpSub, 3)
    st = transfer.rescale_stage(2.5, -1).stages[0]
    assert (st.kind, st.input, st.k[0], st.k[1]) == (vec.OpAffine, -1, 2.5, -1.0)


def test_builder_constants_over_random_options():
    """The stage builders' resolved constants (Horn and ZT scales, the
    hillshade light vector, Gaussian taps) equal the oracle's own
    resolution bit for bit over a seeded sweep of options: cell sizes over
    nine decades, anisotropic cells, negative and fractional z factors,
    azimuths past a full turn and altitudes over the whole range."""
    rng = np.random.default_rng(20261204)
    for _ in range(400):
        cs = float(np.float32(10 ** rng.uniform(-4, 5)))
        csy = 0.0 if rng.random() < 0.4 else float(np.float32(10 ** rng.uniform(-4, 5)))
        z = 0.0 if rng.random() < 0.3 else float(np.float32(rng.uniform(-10, 10)))
        kx, ky = orc.horn_scales(cs, csy or cs, z or 1.0)
        got = k_of(terrain.slope_stage(terrain.SlopeOptions(CellSize=cs, CellSizeY=csy, ZFactor=z)))
        assert (got[0], got[1]) == (kx, ky), (cs, csy, z)
        got = k_of(terrain.curvature_stage(terrain.CurvatureOptions(CellSize=cs, CellSizeY=csy, ZFactor=z, Type=1)))
        assert got[:5] == orc.zt_scales(cs, csy or cs, z or 1.0), (cs, csy, z)
        az, alt = float(np.float32(rng.uniform(-720, 720))), float(np.float32(rng.uniform(0, 90)))
        got = k_of(terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=cs, CellSizeY=csy, ZFactor=z,
                                                                    Azimuth=az, Altitude=alt)))
        assert (got[0], got[1]) == (kx, ky) and got[2:5] == orc.hillshade_light(az, alt), (cs, csy, z, az, alt)
    for r in range(1, 9):
        for sigma in rng.uniform(0.05, 20, 6):
            sigma = float(np.float32(sigma))
            assert (focal.Gaussian(r, sigma).view(np.uint32) == orc.gaussian(r, sigma).view(np.uint32)).all(), (r, sigma)
