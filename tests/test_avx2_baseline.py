"""The restated AVX2 baseline (oracle/strata_avx2.c, after the reference's
internal/stencil/simd_amd64.go) against the scalar oracle: the reference
promises the same bits from its AVX2 lanes as from its scalar kernels
(simd_amd64.go:9-11), so the restatement must give the scalar oracle's bits
on every cell, tails and edge rings included. Also: the oracle's own stage
builders (used where the device library must not load, the benchmark's
reference arm) resolve the options to the product builders' constants."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as orc
from strata_b200 import synth, terrain

from helpers import poison, same_bits

OPS = {
    "gradient": (lambda: orc.gradient_stage(10.0), 2),
    "slope_deg": (lambda: orc.slope_stage(30.0), 1),
    "slope_pct": (lambda: orc.slope_stage(10.0, units=1), 1),
    "slope_rad_aniso": (lambda: orc.slope_stage(3.0, 7.0, 2.0, units=2), 1),
    "aspect": (lambda: orc.aspect_stage(30.0), 1),
    "aspect_trig_zero": (lambda: orc.aspect_stage(5.0, zero_for_flat=True, trigonometric=True), 1),
    "hillshade": (lambda: orc.hillshade_stage(10.0), 1),
    "hillshade_light": (lambda: orc.hillshade_stage(2.0, 3.0, azimuth=97.5, altitude=30.0), 1),
    "curv_profile": (lambda: orc.curvature_stage(10.0, kind=0), 1),
    "curv_plan": (lambda: orc.curvature_stage(10.0, kind=1), 1),
    "curv_mean": (lambda: orc.curvature_stage(3.0, 4.0, kind=2), 1),
    "tri": (lambda: orc.ruggedness_stage(0), 1),
    "wilson": (lambda: orc.ruggedness_stage(1), 1),
    "tpi": (lambda: orc.ruggedness_stage(2), 1),
    "roughness": (lambda: orc.ruggedness_stage(3), 1),
    # wider windows: scalar cells, word-level validity in the baseline's engine
    "tpi_r3": (lambda: orc.ruggedness_stage(2, 3), 1),
    "mean_r8": (lambda: orc.stage(orc.MEAN, 8), 1),
}


def _run(stages, cells, valid, nout, simd, nthreads=2):
    h, w = cells.shape
    src = dict(data=np.ascontiguousarray(cells.reshape(-1)), width=w, height=h, stride=w,
               valid=orc.pack_mask(valid) if valid is not None else None, valid_offset=0)
    outs = []
    for _ in range(nout):
        outs.append(dict(data=np.full(w * h, 7.25, np.float32), width=w, height=h, stride=w,
                         valid=np.zeros((w * h + 63) // 64, np.uint64) if valid is not None else None,
                         valid_offset=0))
    orc.process(stages, src, outs, nthreads, simd=simd)
    return outs


@pytest.mark.parametrize("name", sorted(OPS))
@pytest.mark.parametrize("w,h", [(3, 3), (9, 5), (17, 11), (64, 33), (203, 41)])
def test_avx2_lanes_equal_scalar(name, w, h):
    mk, nout = OPS[name]
    cells = poison(synth.fbm_dem(w, h, w * 31 + h), w + h, 0.02)
    valid = synth.cell_mask(w, h, w + 7 * h, 0.05)
    for v in (None, valid):
        a = _run([mk()], cells, v, nout, simd=False)
        b = _run([mk()], cells, v, nout, simd=True)
        for k in range(nout):
            ok = same_bits(a[k]["data"], b[k]["data"])
            assert ok.all(), f"{name} {w}x{h}: {int((~ok).sum())} cells differ, first at {np.argmin(ok)}"
            if v is not None:
                assert (a[k]["valid"] == b[k]["valid"]).all()


def test_avx2_pipeline_equals_scalar():
    w, h = 517, 37
    cells = synth.fbm_dem(w, h, 5)
    stages = [orc.slope_stage(10.0), orc.lookup_stage([0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5]),
              orc.reclass_stage([1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5])]
    a = _run(stages, cells, None, 1, simd=False)
    b = _run(stages, cells, None, 1, simd=True)
    assert same_bits(a[0]["data"], b[0]["data"]).all()


def _k(stage_and_keep):
    st, _keep = stage_and_keep
    return st.op, st.kind, list(np.float32(st.k[i]) for i in range(5))


@pytest.mark.parametrize("cs", [1.0, 10.0, 30.0, 37.5])
def test_oracle_builders_match_product_builders(cs):
    pairs = [
        (orc.gradient_stage(cs), terrain.gradient_stage(terrain.GradientOptions(CellSize=cs))),
        (orc.slope_stage(cs), terrain.slope_stage(terrain.SlopeOptions(CellSize=cs))),
        (orc.slope_stage(cs, units=1), terrain.slope_stage(terrain.SlopeOptions(CellSize=cs, Units=1))),
        (orc.aspect_stage(cs), terrain.aspect_stage(terrain.AspectOptions(CellSize=cs))),
        (orc.hillshade_stage(cs, azimuth=315, altitude=45),
         terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=cs, Azimuth=315, Altitude=45, ZFactor=1))),
        (orc.curvature_stage(cs, kind=2), terrain.curvature_stage(terrain.CurvatureOptions(CellSize=cs, Type=2))),
    ]
    for o, p in pairs:
        st = p.stages[0]
        want = (st.op, st.kind, [np.float32(st.k[i]) for i in range(5)])
        assert _k(o) == want
