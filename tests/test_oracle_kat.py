"""Pins the oracle (oracle/strata_oracle.c) against the known-answer tests
of the reference's own test suite (tests/golden/kat.json, transcribed by
tests/golden/make_kat.py with the file:line of each case), and against
the reference's accuracy bounds. CPU only."""
from __future__ import annotations

import json
import math
import os
import struct

import numpy as np
import pytest

from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
KAT = json.load(open(os.path.join(HERE, "golden", "kat.json")))


def f(h: str) -> np.float32:
    return np.array([int(h, 16)], np.uint32).view(np.float32)[0]


def fs(hs):
    return np.array([int(h, 16) for h in hs], np.uint32).view(np.float32)


def bits(x) -> int:
    return int(np.array([x], np.float32).view(np.uint32)[0])


def same(a, b) -> bool:
    a, b = np.float32(a), np.float32(b)
    return (np.isnan(a) and np.isnan(b)) or bits(a) == bits(b)


def raster(cells, w, h, valid=None):
    d = np.ascontiguousarray(np.asarray(cells, np.float32).reshape(-1))
    return dict(data=d, width=w, height=h, stride=w, valid=valid, valid_offset=0)


def run(stages, src, ndst=1):
    outs = [raster(np.zeros(src["width"] * src["height"]), src["width"], src["height"]) for _ in range(ndst)]
    orc.process(stages, src, outs)
    return [o["data"] for o in outs]


def horn_k(cs):
    kx, ky = orc.horn_scales(cs, cs, 1.0)
    return kx, ky


# ---------------------------------------------------------------------------
# Arctangents.

def test_atan32_specials():
    for x, want in KAT["atan32_exact"]["rows"]:
        assert bits(orc.atan32(f(x))) == int(want, 16)
    assert np.isnan(orc.atan32(np.float32("nan")))


def test_atan32_accuracy_stride():
    """TestAtan32Accuracy (internal/stencil/stencil_test.go:9-34): every
    9973rd non-negative finite bit pattern within 1.5e-7 of math.Atan, and
    the 2000 floats around tan(pi/8), tan(3pi/8) and 1."""
    b = np.arange(0, 0x7F800000, 9973, dtype=np.uint32)
    x = b.view(np.float32)
    got = orc.atan32_array(x).astype(np.float64)
    err = np.abs(got - np.arctan(x.astype(np.float64)))
    assert err.max() <= 1.5e-7, err.max()
    for th in (np.float32(0.4142135623730950), np.float32(2.414213562373095), np.float32(1.0)):
        base = int(np.array([th], np.float32).view(np.uint32)[0])
        xs = np.arange(base - 1000, base + 1000, dtype=np.uint32).view(np.float32)
        g = orc.atan32_array(xs).astype(np.float64)
        assert np.abs(g - np.arctan(xs.astype(np.float64))).max() <= 1.5e-7


def test_atan32_monotone_on_nonnegative_floats():
    """Atan32 never falls as its argument grows, over every non-negative
    float up to +Inf. The device backend classifies a Slope by its squared
    gradient magnitude (api.cu fold_slope_square) on the strength of this."""
    assert orc.atan32_drops(os.cpu_count() or 1) == 0


def test_atan2f32_exact_table():
    for y, x, want in KAT["atan2f32_exact"]["rows"]:
        got = orc.atan2f32(f(y), f(x))
        assert bits(got) == int(want, 16), (y, x, hex(bits(got)), want)


def test_atan2f32_accuracy():
    """TestAtan2F32Accuracy (stencil_test.go:348-384): special pairs and a
    random sample within 3e-7 of math.Atan2, with math.Atan2's sign."""
    sp = fs(KAT["atan2_specials"]["values"])
    ys, xs = np.meshgrid(sp, sp, indexing="ij")
    rng = np.random.default_rng(21)
    n = 200_000

    def sample(k):
        v = np.where(rng.integers(0, 4, k) == 0, rng.random(k) * 4, 2.0 ** (rng.random(k) * 200 - 100))
        return (v * np.where(rng.integers(0, 2, k) == 0, -1, 1)).astype(np.float32)

    ry, rx = sample(n), sample(n)
    near = (np.nextafter(ry, np.float32(0)) * np.where(rng.integers(0, 2, n) == 0, 1, -1)).astype(np.float32)
    Y = np.concatenate([ys.ravel(), ry, ry])
    X = np.concatenate([xs.ravel(), rx, near])
    got = orc.atan2f32_array(Y, X)
    want = np.arctan2(Y.astype(np.float64), X.astype(np.float64))
    nan = np.isnan(want)
    assert np.isnan(got[nan]).all()
    ok = ~nan
    assert (np.signbit(got[ok]) == np.signbit(want[ok])).all()
    assert np.abs(got[ok].astype(np.float64) - want[ok]).max() <= KAT["atan2_specials"]["bound"]


def test_go_min_max_pairs():
    """Go's builtin min / max over every ordered pair of special values: NaN
    wins, -0 orders below +0 (the rule TestSIMDMinMaxEdgePairs pins,
    internal/focalrow/simd_test.go)."""
    vals = [np.float32(v) for v in (0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 1e-45, -3e38)]
    for a in vals:
        for b in vals:
            lo, hi = orc.go_min(a, b), orc.go_max(a, b)
            if np.isnan(a) or np.isnan(b):
                assert np.isnan(lo) and np.isnan(hi)
                continue
            if a == b == 0:
                neg_a, neg_b = np.signbit(a), np.signbit(b)
                assert np.signbit(lo) == (neg_a or neg_b)
                assert np.signbit(hi) == (neg_a and neg_b)
                continue
            assert lo == min(float(a), float(b)) and hi == max(float(a), float(b))


# ---------------------------------------------------------------------------
# Ruggedness, terrain and focal known answers.

@pytest.mark.parametrize("row", KAT["ruggedness_windows"]["rows"], ids=lambda r: r["name"])
def test_ruggedness_known_windows(row):
    src = raster(fs(row["w"]), 3, 3)
    for kind, want in enumerate(row["want"]):
        (out,) = run([orc.stage(orc.RUGGEDNESS, 1, kind)], src)
        assert bits(out[4]) == int(want, 16), (row["name"], kind, out[4])


def test_roughness_nan_and_signed_zero():
    c = KAT["roughness_special"]
    (out,) = run([orc.stage(orc.RUGGEDNESS, 1, 3)], raster(fs(c["nan_window"]), 3, 3))
    assert np.isnan(out[4])
    (out,) = run([orc.stage(orc.RUGGEDNESS, 1, 3)], raster(fs(c["zero_window"]), 3, 3))
    assert bits(out[4]) == int(c["zero_want"], 16)


def test_slope_esri_hand_computed():
    c = KAT["slope_esri"]
    src = raster(fs(c["dem"]), 3, 3)
    kx, ky = horn_k(c["cell_size"])
    dx, dy = run([orc.stage(orc.GRADIENT, 1, 0, [kx, ky])], src, 2)
    assert abs(float(dx[4]) - c["dx"]) <= c["grad_tol"]
    assert abs(float(dy[4]) - c["dy"]) <= c["grad_tol"]
    scales = {0: (np.float32(180 / math.pi), 1), 1: (np.float32(100), 0), 2: (np.float32(1), 1)}
    for units, want, tol in c["units"]:
        scale, atan = scales[units]
        (out,) = run([orc.stage(orc.SLOPE, 1, atan, [kx, ky, scale])], src)
        assert abs(float(out[4]) - want) <= tol, (units, out[4], want)
        assert np.isnan(np.delete(out, 4)).all()


def test_flat_is_zero():
    """TestFlatIsZero (terrain/terrain_test.go:109-123): +0 in every unit."""
    src = raster(np.full(12 * 5, 1234.5), 12, 5)
    kx, ky = horn_k(30)
    for scale, atan in ((np.float32(180 / math.pi), 1), (np.float32(100), 0), (np.float32(1), 1)):
        (out,) = run([orc.stage(orc.SLOPE, 1, atan, [kx, ky, scale])], src)
        inner = out.reshape(5, 12)[1:-1, 1:-1]
        assert (inner.view(np.uint32) == 0).all()


def test_aspect_esri_hand_computed():
    c = KAT["aspect_esri"]
    kx, ky = horn_k(c["cell_size"])
    (out,) = run([orc.stage(orc.ASPECT, 1, 0, [kx, ky, -1])], raster(fs(c["dem"]), 3, 3))
    assert abs(float(out[4]) - c["want"]) <= c["tol"]


def test_hillshade_esri_hand_computed():
    c = KAT["hillshade_esri"]
    kx, ky = horn_k(c["cell_size"])
    src = raster(fs(c["dem"]), 3, 3)
    light = orc.hillshade_light(0, 0)
    (out,) = run([orc.stage(orc.HILLSHADE, 1, 0, [kx, ky] + light)], src)
    assert bits(out[4]) == int(c["default_light_want"], 16)
    light = orc.hillshade_light(90, 0)
    (out,) = run([orc.stage(orc.HILLSHADE, 1, 0, [kx, ky] + light)], src)
    assert abs(float(out[4]) - c["azimuth_90_want"]) <= c["tol"]


def test_curvature_hand_computed():
    c = KAT["curvature_hand"]
    k = orc.zt_scales(1, 1, 1)
    for kind, want in c["want"]:
        (out,) = run([orc.stage(orc.CURVATURE, 1, kind, k)], raster(fs(c["dem"]), 3, 3))
        assert abs(float(out[4]) - want) <= c["rel_tol"] * abs(want)


def test_curvature_flat_and_plane_masked():
    """TestCurvatureFlatAndPlane (terrain/curvature_test.go:156-182): +0 and
    valid everywhere inside, for a flat DEM and a plane."""
    w, h = 8, 6
    flat = np.full(w * h, 812.25, np.float32)
    y, x = np.mgrid[0:h, 0:w]
    plane = (3 * x - 2 * y + 1).astype(np.float32).reshape(-1)
    for dem in (flat, plane):
        valid = np.full(1, (1 << 48) - 1, np.uint64)
        for cs, csy, z in ((1, 1, 1), (3, 0.5, -2)):
            k = orc.zt_scales(cs, csy, z)
            for kind in range(3):
                src = raster(dem, w, h, valid)
                out = raster(np.zeros(w * h), w, h, np.zeros(1, np.uint64))
                orc.process([orc.stage(orc.CURVATURE, 1, kind, k)], src, [out])
                inner = out["data"].reshape(h, w)[1:-1, 1:-1]
                assert (inner.view(np.uint32) == 0).all()
                vb = [(int(out["valid"][0]) >> (yy * w + xx)) & 1 for yy in range(h) for xx in range(w)]
                vb = np.array(vb).reshape(h, w)
                assert vb[1:-1, 1:-1].all() and vb[0].sum() == 0 and vb[:, 0].sum() == 0


def test_curvature_nan_centre():
    for c in (np.nan, np.inf, -np.inf):
        for kind in range(3):
            (out,) = run([orc.stage(orc.CURVATURE, 1, kind, orc.zt_scales(1, 1, 1))],
                         raster([5, 5, 5, 5, c, 5, 5, 5, 5], 3, 3))
            if kind == 2 and not np.isnan(c):
                assert np.isinf(out[4])
            else:
                assert np.isnan(out[4])


def test_focal_hand_computed():
    c = KAT["focal_hand"]
    src = raster(fs(c["src"]), 3, 3)
    w = fs(c["weights"])
    checks = [
        ([orc.stage(orc.CORRELATE, 1, 0, [], [w])], c["correlate"]),
        ([orc.stage(orc.CORRELATE, 1, 0, [], [w[::-1].copy()])], c["convolve"]),
        ([orc.stage(orc.SEPARABLE, 1, 0, [], [fs(c["separable_shift"]["row"]), fs(c["separable_shift"]["col"])])],
         c["separable_shift"]["want"]),
        ([orc.stage(orc.SEPARABLE, 1, 0, [], [fs(c["separable_sums"]["row"]), fs(c["separable_sums"]["col"])])],
         c["separable_sums"]["want"]),
        ([orc.stage(orc.MEAN, 1)], c["mean"]),
        ([orc.stage(orc.MIN, 1)], c["min"]),
        ([orc.stage(orc.MAX, 1)], c["max"]),
    ]
    for stages, want in checks:
        (out,) = run(stages, src)
        assert bits(out[4]) == int(want, 16), (stages[0][0].op, out[4])
        assert np.isnan(np.delete(out, 4)).all()


def test_focal_signed_zero():
    """TestSignedZero (focal/focal_test.go:219-246): sums of -0 stay -0."""
    src = raster(np.full(120, -0.0, np.float32), 40, 3)
    one9 = np.ones(9, np.float32)
    one3 = np.ones(3, np.float32)
    for st in (orc.stage(orc.CORRELATE, 1, 0, [], [one9]), orc.stage(orc.SEPARABLE, 1, 0, [], [one3, one3]),
               orc.stage(orc.MEAN, 1), orc.stage(orc.MIN, 1), orc.stage(orc.MAX, 1)):
        (out,) = run([st], src)
        row = out.reshape(3, 40)[1, 1:39]
        assert (row.view(np.uint32) == 0x80000000).all()


# ---------------------------------------------------------------------------
# Lookup and Reclass.

def pointwise(stage, src):
    s = fs(src)
    (out,) = run([stage], raster(s, len(s), 1))
    return out


@pytest.mark.parametrize("i", range(len(KAT["reclass"]["rows"])))
def test_reclass_known(i):
    r = KAT["reclass"]["rows"][i]
    out = pointwise(orc.stage(orc.RECLASS, 0, 0, [], [fs(r["breaks"]), fs(r["values"])]), r["src"])
    for g, w in zip(out, fs(r["want"])):
        assert same(g, w), (g, w)


@pytest.mark.parametrize("i", range(len(KAT["lookup"]["rows"])))
def test_lookup_known(i):
    r = KAT["lookup"]["rows"][i]
    out = pointwise(orc.stage(orc.LOOKUP, 0, 0, [], [fs(r["xs"]), fs(r["ys"])]), r["src"])
    for g, w in zip(out, fs(r["want"])):
        assert same(g, w), (g, w)


def test_lookup_not_fused():
    c = KAT["lookup_not_fused"]
    out = pointwise(orc.stage(orc.LOOKUP, 0, 0, [], [fs(c["xs"]), fs(c["ys"])]), [c["src"]])
    assert bits(out[0]) == int(c["want"], 16)


def test_knots_exact():
    c = KAT["knots_exact"]
    out = pointwise(orc.stage(orc.LOOKUP, 0, 0, [], [fs(c["xs"]), fs(c["ys"])]), c["xs"])
    for g, w in zip(out, fs(c["ys"])):
        assert same(g, w)


def test_nan_payload_kept():
    src = KAT["nan_payload"]["src"]
    for st in (orc.stage(orc.RECLASS, 0, 0, [], [fs(["0x00000000"]), fs(["0x3f800000", "0x40000000"])]),
               orc.stage(orc.LOOKUP, 0, 0, [], [fs(["0x00000000", "0x3f800000"]), fs(["0x3f800000", "0x40000000"])])):
        out = pointwise(st, src)
        assert [hex(bits(v)) for v in out] == [hex(int(s, 16)) for s in src]


# ---------------------------------------------------------------------------
# Engine rules.

def test_validity_erosion_matches_naive():
    """Output validity = the window's AND, edge ring cleared
    (internal/exec/halo.go:213-229), against a naive per-cell count, with a
    stride and a bit offset."""
    rng = np.random.default_rng(5)
    for r in (1, 2, 5):
        w, h, stride, off = 37, 23, 41, 13
        valid = rng.random((h, w)) > 0.03
        bitsarr = np.zeros(((off + (h - 1) * stride + w + 63) // 64) * 64, np.uint8)
        for yy in range(h):
            bitsarr[off + yy * stride:off + yy * stride + w] = valid[yy]
        m = np.packbits(bitsarr, bitorder="little").view(np.uint64).copy()
        data = rng.random((h - 1) * stride + w).astype(np.float32)
        src = dict(data=data, width=w, height=h, stride=stride, valid=m, valid_offset=off)
        dm = np.zeros_like(m)
        dst = dict(data=np.zeros_like(data), width=w, height=h, stride=stride, valid=dm, valid_offset=off)
        orc.process([orc.stage(orc.MEAN, r)], src, [dst])
        got = np.unpackbits(dm.view(np.uint8), bitorder="little")
        for yy in range(h):
            for xx in range(w):
                want = (r <= xx < w - r and r <= yy < h - r and valid[yy - r:yy + r + 1, xx - r:xx + r + 1].all())
                assert bool(got[off + yy * stride + xx]) == want


def test_reclass_without_breaks():
    """Zero breaks: every cell takes the one value, NaN stays NaN."""
    out = pointwise(orc.stage(orc.RECLASS, 0, 0, [], [np.zeros(0, np.float32), fs(["0x40e00000"])]),
                    ["0x7fc00000", "0xbf800000", "0x80000000", "0x7f800000"])
    assert np.isnan(out[0]) and (out[1:] == np.float32(7)).all()


def test_pointwise_tables_checked():
    """Mismatched or missing Lookup / Reclass tables are an invalid call,
    not a read past them."""
    src = raster([1, 2, 3], 3, 1)
    bad = [orc.stage(orc.RECLASS, 0, 0, [], [fs(["0x3f800000"])]),
           orc.stage(orc.RECLASS, 0, 0, [], [fs(["0x3f800000"]), fs(["0x3f800000"])]),
           orc.stage(orc.LOOKUP, 0, 0, [], [fs(["0x3f800000", "0x40000000"]), fs(["0x3f800000"])]),
           orc.stage(orc.LOOKUP, 0, 0, [], [])]
    for st in bad:
        with pytest.raises(ValueError):
            run([st], src)


# ---------------------------------------------------------------------------
# HeatLoad, Orientation and Wood's fit (terrain/heatload.go, orientation.go,
# fit.go): the reference's known answers and closed forms.

def _run1(stage, cells, nout=1):
    h, w = cells.shape
    src = dict(data=np.ascontiguousarray(cells, np.float32).reshape(-1), width=w, height=h, stride=w, valid=None,
               valid_offset=0)
    outs = [dict(data=np.full(w * h, 7.0, np.float32), width=w, height=h, stride=w, valid=None, valid_offset=0)
            for _ in range(nout)]
    orc.process([stage], src, outs)
    return [o["data"].reshape(h, w) for o in outs]


def _plane(w, h, a, b_, cs=1.0, csy=1.0):
    """terrain/terrain_test.go:28-36: z = a*x*cs + b*y*csy + 100, as float32."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    return (a * x * cs + b_ * y * csy + 100).astype(np.float32)


def test_heatload_mccune_keon_table():
    """TestHeatLoadMcCuneKeon (terrain/heatload_test.go:66-109): all 36
    values of the authors' spreadsheet and the arithmetic-scale column."""
    case = KAT["heatload_mccune_keon"]
    for lat, slope, aspect, rad, heat in case["rows"]:
        t = math.tan(slope * math.pi / 180) * (-1 if aspect == 180 else 1)
        dem = np.array([[t * y for _x in range(5)] for y in range(5)], np.float32)
        for eq in range(3):
            for radiation in (True, False):
                want = (rad if radiation else heat)[eq]
                for linear in (False, True):
                    w = math.exp(want) if linear and eq < 2 else want
                    (got,) = _run1(orc.heatload_stage(1.0, latitude=lat, equation=eq, radiation=radiation,
                                                      linear=linear), dem)
                    assert np.isnan(got[0]).all() and np.isnan(got[:, 0]).all()
                    inner = got[1:-1, 1:-1].astype(np.float64)
                    assert np.abs(inner - w).max() <= case["tol"], (lat, slope, aspect, eq, radiation, linear)


def test_orientation_cardinal_exact():
    """TestOrientationCardinal (terrain/orientation_test.go:76-101)."""
    for row in KAT["orientation_cardinal"]["rows"]:
        dem = _plane(5, 5, row["a"], row["b"])
        for unweighted in (True, False):
            for east, key in ((False, "north"), (True, "east")):
                (got,) = _run1(orc.orientation_stage(1.0, east=east, unweighted=unweighted), dem)
                want = f(row[key] if unweighted else row[key + "W"])
                assert got[2, 2] == want, (row, east, unweighted, got[2, 2], want)


def test_orientation_planes():
    """TestOrientationPlanes (terrain/orientation_test.go:41-74): the eight
    compass directions at four steepnesses against the closed form."""
    for da, db in ((0, 1), (1, 1), (1, 0), (1, -1), (0, -1), (-1, -1), (-1, 0), (-1, 1)):
        for steep in (0.05, 0.5, 1, 4):
            a, b_ = da * steep, db * steep
            dem = _plane(7, 6, a, b_, 10, 10)
            for east in (False, True):
                for unweighted in (False, True):
                    comp = -a if east else b_
                    want = comp / (math.hypot(a, b_) if unweighted else math.sqrt(1 + a * a + b_ * b_))
                    (got,) = _run1(orc.orientation_stage(10.0, east=east, unweighted=unweighted), dem)
                    assert np.abs(got[1:-1, 1:-1] - want).max() <= 1e-6


def test_fit_plane():
    """TestFitPlane (terrain/fit_test.go:36-72): on a plane the fit's
    gradient is the plane's and every curvature is +0, edges NaN."""
    for a, b_ in ((0, 0), (1, 0), (0, -3), (2, 5), (-7, 4)):
        for r in range(1, 9):
            dem = _plane(2 * r + 5, 2 * r + 4, a, b_)
            gx, gy = _run1(orc.fit_stage(orc.GRADIENT, r, 1.0), dem, 2)
            inner = (slice(r, -r), slice(r, -r))
            assert np.isnan(gx[:r]).all() and np.isnan(gy[:, :r]).all()
            assert np.abs(gx[inner] - a).max() <= 1e-6 * abs(a)
            assert np.abs(gy[inner] - b_).max() <= 1e-6 * abs(b_)
            for kind in range(3):
                (cv,) = _run1(orc.fit_stage(orc.CURVATURE, r, 1.0, kind=kind), dem)
                assert (cv[inner].view(np.uint32) == 0).all(), (a, b_, r, kind)


def test_fit_quadratic():
    """TestFitQuadratic (terrain/fit_test.go:74-132): least squares fits a
    quadratic exactly, so the fit's gradient and curvatures are the
    surface's, within the float32 rounding of the elevations' sums."""
    w, h = 40, 36
    cx, cy, zf = 2.0, 3.0, 1.5
    c = (0.03, -0.02, 0.01, 0.4, -0.25, 50)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    X, Y = xx * cx, yy * cy
    dem = (c[0] * X * X + c[1] * Y * Y + c[2] * X * Y + c[3] * X + c[4] * Y + c[5]).astype(np.float32)
    zmax = float(np.abs(dem).max())
    for r in (1, 2, 4, 8):
        gx, gy = _run1(orc.fit_stage(orc.GRADIENT, r, cx, cy, zf), dem, 2)
        k = 2 * r + 1
        e = 4 * k * k * zmax * 2.0 ** -24
        s2 = r * (r + 1) * (2 * r + 1) / 3
        inner = (slice(r, h - r), slice(r, w - r))
        p = zf * (2 * c[0] * X + c[2] * Y + c[3])[inner]
        q = zf * (2 * c[1] * Y + c[2] * X + c[4])[inner]
        assert (np.abs(gx[inner] - p) <= zf * e * r * k / (k * s2 * cx) + 1e-6 * np.abs(p)).all()
        assert (np.abs(gy[inner] - q) <= zf * e * r * k / (k * s2 * cy) + 1e-6 * np.abs(q)).all()
        rr, tt, ss = zf * 2 * c[0], zf * 2 * c[1], zf * c[2]
        g = p * p + q * q
        want = [-(p * p * rr + 2 * p * q * ss + q * q * tt) / (g * (1 + g) ** 1.5),
                -(q * q * rr - 2 * p * q * ss + p * p * tt) / g ** 1.5,
                -((1 + q * q) * rr - 2 * p * q * ss + (1 + p * p) * tt) / (2 * (1 + g) ** 1.5)]
        for kind in range(3):
            (cv,) = _run1(orc.fit_stage(orc.CURVATURE, r, cx, cy, zf, kind=kind), dem)
            got = cv[inner].astype(np.float64)
            assert (np.abs(got - want[kind]) <= 2e-3 * np.abs(want[kind]) + 1e-6).all(), (r, kind)
