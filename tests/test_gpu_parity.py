"""Device parity: every op of the path through libstrata_cuda against the
oracle on the same seeded inputs, cell for cell (rastertest.SameFloat:
same bits, or both NaN) and bit for bit in the validity masks, over the
shapes, layouts and masks of the reference's engine matrix
(internal/exec/workers_test.go:29-80): tiny and odd shapes, strided
windows with bit offsets, unmasked / masked inputs and masked outputs of
unmasked inputs, host-memory and device-resident operands."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from helpers import (assert_padding_untouched, assert_same_raster, host_raster, like, poison, run_oracle,
                     to_device, to_host)
from strata_b200 import engine, focal, synth, terrain, transfer
from strata_b200.raster import Float32Raster

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 5), (3, 3), (4, 4), (17, 5), (61, 37), (300, 9), (129, 67), (257, 131), (516, 70), (1028, 33)]
SMALL_SHAPES = [(3, 3), (4, 9), (19, 23), (61, 37), (128, 40), (132, 21)]


def dem_cells(w, h, seed):
    return poison(synth.fbm_dem(w, h, seed, lo=0, hi=3000), seed, 0.003)


def focal_cells(w, h, seed):
    return poison(synth.normal_trend(w, h, seed), seed, 0.003)


def layouts(w, h, seed, masked):
    """(src, dst) pairs: compact; strided with bit offsets; masked output
    of an unmasked input."""
    out = []
    valid = synth.cell_mask(w, h, seed, 0.03) if masked else None
    yield dict(src=dict(stride=None, offset=0, valid=valid), dst=dict(stride=None, offset=0, masked=masked))
    yield dict(src=dict(stride=w + 13, offset=37, valid=valid), dst=dict(stride=w + 5, offset=11, masked=masked))
    yield dict(src=dict(stride=w + 8, offset=5, valid=valid), dst=dict(stride=w + 4, offset=70, masked=masked))
    if not masked:
        yield dict(src=dict(stride=w + 1, offset=0, valid=None), dst=dict(stride=None, offset=63, masked=True))


def check_case(stages, cells, nout=1, device=False, lay=None, what=""):
    h, w = cells.shape
    src = host_raster(cells, lay["src"]["valid"], lay["src"]["stride"], lay["src"]["offset"])
    want = [like(src, lay["dst"]["stride"], lay["dst"]["offset"], masked=lay["dst"]["masked"]) for _ in range(nout)]
    got = [like(src, lay["dst"]["stride"], lay["dst"]["offset"], masked=lay["dst"]["masked"]) for _ in range(nout)]
    before = [Float32Raster(np.array(g.data), g.width, g.height, g.stride,
                            None if g.valid is None else np.array(g.valid), g.valid_offset) for g in got]
    run_oracle(stages, src, want)
    if device:
        dsrc = to_device(src)
        dgot = [to_device(g) for g in got]
        assert engine.process(stages, dgot, [dsrc]) is None
        got = [to_host(g) for g in dgot]
    else:
        assert engine.process(stages, got, [src]) is None
    for i in range(nout):
        assert_same_raster(got[i], want[i], f"{what} out{i}")
        assert_padding_untouched(before[i], got[i], f"{what} out{i}")


def run_matrix(make_stages, cells_fn, nout=1, shapes=SHAPES, seed=1):
    for (w, h), masked, device in itertools.product(shapes, (False, True), (False, True)):
        cells = cells_fn(w, h, seed + w * 7 + h)
        for li, lay in enumerate(layouts(w, h, seed + w + h, masked)):
            check_case(make_stages(), cells, nout, device, lay,
                       f"{w}x{h} masked={masked} device={device} layout={li}")


TERRAIN = {
    "slope_deg": lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=30)),
    "slope_pct": lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10, Units=terrain.SlopePercent)),
    "slope_rad_aniso": lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=3, CellSizeY=7, ZFactor=2,
                                                                        Units=terrain.SlopeRadians)),
    "aspect": lambda: terrain.aspect_stage(terrain.AspectOptions(CellSize=30)),
    "aspect_trig_zero": lambda: terrain.aspect_stage(terrain.AspectOptions(CellSize=5, ZeroForFlat=True,
                                                                           Trigonometric=True)),
    "hillshade": lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10)),
    "hillshade_light": lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=2, CellSizeY=3,
                                                                                Azimuth=97.5, Altitude=30)),
    "curv_profile": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=0)),
    "curv_plan": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=1)),
    "curv_mean": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=3, CellSizeY=4, Type=2)),
}


@pytest.mark.parametrize("name", sorted(TERRAIN))
def test_terrain_ops(name):
    run_matrix(TERRAIN[name], dem_cells)


def gentle_cells(w, h, seed):
    """Gentle terrain (slopes mostly below 22.5 degrees, where whole warps
    skip the arctangent's division) with a few steep ridges and scattered
    special values, so warps that skip and warps that divide both occur,
    and some warps mix both kinds of lanes."""
    cells = synth.fbm_dem(w, h, seed, lo=0, hi=3000) * np.float32(0.01)
    rng = np.random.default_rng(seed)
    for _ in range(max(1, w * h // 4000)):
        y, x = int(rng.integers(0, h)), int(rng.integers(0, w))
        cells[y, x:x + int(rng.integers(1, 40))] += np.float32(rng.uniform(5, 400))
    return poison(cells.astype(np.float32), seed, 0.001)


@pytest.mark.parametrize("units", ["deg", "rad"])
def test_slope_on_gentle_terrain(units):
    """Slope with the arctangent over gentle terrain: the warps whose
    magnitudes all lie below tan(pi/8) take the arctangent without its
    division, the others with it; every cell matches the oracle."""
    u = terrain.SlopeDegrees if units == "deg" else terrain.SlopeRadians
    run_matrix(lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10, Units=u)), gentle_cells,
               shapes=[(257, 131), (516, 70), (1028, 33), (2052, 40)], seed=7)


def test_gradient_two_outputs():
    run_matrix(lambda: terrain.gradient_stage(terrain.GradientOptions(CellSize=30, CellSizeY=25)), dem_cells, nout=2)


@pytest.mark.parametrize("kind", range(4))
@pytest.mark.parametrize("r", [1, 2, 3, 5, 8])
def test_ruggedness(kind, r):
    run_matrix(lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=kind, Radius=r)), dem_cells,
               shapes=SMALL_SHAPES, seed=kind * 10 + r)


@pytest.mark.parametrize("r", range(1, 9))
def test_correlate(r):
    w = synth.uniform_weights((2 * r + 1) ** 2, r)
    run_matrix(lambda: focal.weights_stage(focal.WeightsOptions(Radius=r, Weights=w), False), focal_cells,
               shapes=SMALL_SHAPES, seed=r)


@pytest.mark.parametrize("r", [1, 3, 8])
def test_convolve(r):
    w = synth.uniform_weights((2 * r + 1) ** 2, 100 + r)
    run_matrix(lambda: focal.weights_stage(focal.WeightsOptions(Radius=r, Weights=w), True), focal_cells,
               shapes=SMALL_SHAPES, seed=r)


@pytest.mark.parametrize("r", range(1, 9))
def test_separable(r):
    row = synth.uniform_weights(2 * r + 1, 200 + r)
    col = focal.Gaussian(r, 2.5)
    run_matrix(lambda: focal.separable_stage(focal.SeparableOptions(Radius=r, Row=row, Col=col)), focal_cells,
               shapes=SMALL_SHAPES, seed=r)


@pytest.mark.parametrize("op", ["mean", "min", "max"])
@pytest.mark.parametrize("r", range(1, 9))
def test_box(op, r):
    opc = {"mean": engine._lib.OP_MEAN, "min": engine._lib.OP_MIN, "max": engine._lib.OP_MAX}[op]
    run_matrix(lambda: focal.box_stage(focal.BoxOptions(Radius=r), opc), focal_cells, shapes=SMALL_SHAPES, seed=r)


SLOPE_XS, SLOPE_YS = [0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5]
BREAKS, VALUES = [1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5]


def test_lookup_and_reclass():
    def cells(w, h, seed):
        return poison((synth.normal_trend(w, h, seed) * 15 + 20).astype(np.float32), seed, 0.01)

    run_matrix(lambda: transfer.lookup_stage(SLOPE_XS, SLOPE_YS), cells)
    run_matrix(lambda: transfer.reclass_stage(BREAKS, VALUES), cells)


def _near(vals, ulps=40):
    """Every float within ulps of each value, stepping through the floats
    in order (-0 next to +0)."""
    out = []
    for v in np.asarray(vals, np.float32):
        if not np.isfinite(v):
            continue
        b = int(np.array([v], np.float32).view(np.uint32)[0])
        key = (b | 0x80000000) if b < 0x80000000 else (~b & 0xFFFFFFFF)
        keys = np.arange(key - ulps, key + ulps + 1, dtype=np.int64).clip(0x00800000, 0xFF7FFFFF)
        bits = np.where(keys >= 0x80000000, keys & 0x7FFFFFFF, ~keys & 0xFFFFFFFF)
        out.append(bits.astype(np.uint32).view(np.float32))
    return np.concatenate(out) if out else np.zeros(0, np.float32)


def _tail_cells(xs, ys, breaks, seed):
    """Cells on and around every knot, every break's preimage under the
    lookup (where the class changes), ±0, infinities, NaN and random floats."""
    rng = np.random.default_rng(seed)
    pre = []
    for k in range(len(xs) - 1):
        x0, x1, y0, y1 = float(xs[k]), float(xs[k + 1]), float(ys[k]), float(ys[k + 1])
        if y1 != y0:
            for b in breaks:
                t = (float(b) - y0) / (y1 - y0)
                if 0 <= t <= 1:
                    pre.append(x0 + t * (x1 - x0))
    vals = np.concatenate([_near(xs), _near(pre), _near(breaks), _near([0.0], 8),
                           np.array([np.inf, -np.inf, np.nan, 1e30, -1e30], np.float32),
                           rng.standard_normal(4000).astype(np.float32) * float(np.abs(xs).max() + 1),
                           rng.integers(0, 2**32, 2000, dtype=np.uint64).astype(np.uint32).view(np.float32)])
    w = 257
    h = (len(vals) + w - 1) // w
    cells = np.full(w * h, 1.5, np.float32)
    cells[:len(vals)] = vals
    return cells.reshape(h, w)


@pytest.mark.parametrize("seed", range(6))
def test_folded_pointwise_tail_edges(seed):
    """A Lookup followed by Reclass stages (and Reclass stages alone) runs as
    one folded Reclass table on the device; on cells at and around every
    knot, every class threshold, ±0, ±inf and NaN it equals the oracle's
    stages run one after another, bit for bit."""
    rng = np.random.default_rng(100 + seed)
    nk = int(rng.integers(2, 9))
    xs = np.sort(rng.choice(np.arange(-50, 50), nk, replace=False)).astype(np.float32) * np.float32(0.37)
    ys = (rng.standard_normal(nk) * 10).astype(np.float32)  # segments rise and fall
    nb = int(rng.integers(1, 7))
    breaks = np.sort(rng.choice(np.arange(-30, 30), nb, replace=False)).astype(np.float32) * np.float32(0.71)
    values = (rng.standard_normal(nb + 1) * 3).astype(np.float32)
    if seed % 2:
        values[int(rng.integers(nb + 1))] = np.nan  # a NoData class
    breaks2 = np.sort(values[np.isfinite(values)])[:2] + np.float32(0.25)
    breaks2 = np.unique(breaks2)
    values2 = np.arange(len(breaks2) + 1, dtype=np.float32) * 10
    chains = {
        "lookup_reclass": lambda: transfer.lookup_stage(xs, ys).extend(transfer.reclass_stage(breaks, values)),
        "lookup_reclass_reclass": lambda: transfer.lookup_stage(xs, ys).extend(
            transfer.reclass_stage(breaks, values)).extend(transfer.reclass_stage(breaks2, values2)),
        "reclass_reclass": lambda: transfer.reclass_stage(breaks, values).extend(
            transfer.reclass_stage(breaks2, values2)),
    }
    cells = _tail_cells(xs, ys, breaks, seed)
    h, w = cells.shape
    for name, make in chains.items():
        for device in (False, True):
            lay = dict(src=dict(stride=None, offset=0, valid=synth.cell_mask(w, h, seed, 0.05)),
                       dst=dict(stride=None, offset=0, masked=True))
            check_case(make(), cells, 1, device, lay, f"{name} seed={seed} device={device}")
    # after a stencil, in the marching kernel's epilogue
    dem = dem_cells(300, 200, seed) * np.float32(0.05)
    lay = dict(src=dict(stride=None, offset=0, valid=None), dst=dict(stride=None, offset=0, masked=False))
    check_case(terrain.slope_stage(terrain.SlopeOptions(CellSize=1)).extend(
        transfer.lookup_stage(xs, ys)).extend(transfer.reclass_stage(breaks, values)), dem, 1, True, lay,
        f"slope+tail seed={seed}")


@pytest.mark.parametrize("trig", [False, True])
def test_aspect_special_gradients(trig):
    """Aspect where the gradient is zero (flat patches: the flat value),
    where both components overflow to infinity (huge steps: atan2's pi/4
    case, in every quadrant) or one does, and on ±0 and NaN cells, equal to
    the oracle bit for bit."""
    w, h = 96, 64
    rng = np.random.default_rng(7 + trig)
    dem = (rng.standard_normal((h, w)) * 50 + 500).astype(np.float32)
    dem[5:15, 5:30] = np.float32(250.0)  # flat
    dem[20:24, 40:44] = np.float32(-0.0)
    dem[20:24, 44:48] = np.float32(0.0)
    big = np.float32(3e38)
    for k, (sy, sx) in enumerate([(1, 1), (1, -1), (-1, 1), (-1, -1)]):
        y0, x0 = 30 + 8 * (k // 2), 8 + 20 * (k % 2)
        block = np.zeros((5, 5), np.float32)
        block += np.arange(5, dtype=np.float32)[None, :] * (sx * big)
        block += np.arange(5, dtype=np.float32)[:, None] * (sy * big)
        dem[y0:y0 + 5, x0:x0 + 5] = np.nan_to_num(block, posinf=np.inf, neginf=-np.inf)
    dem[50:55, 60:65] = np.arange(5, dtype=np.float32)[None, :] * big  # x only
    dem[3, 70] = np.nan
    make = lambda: terrain.aspect_stage(terrain.AspectOptions(CellSize=10, ZeroForFlat=not trig,
                                                              Trigonometric=trig))
    for masked, device in itertools.product((False, True), (False, True)):
        for li, lay in enumerate(layouts(w, h, 3, masked)):
            check_case(make(), dem, 1, device, lay, f"trig={trig} masked={masked} device={device} layout={li}")


@pytest.mark.parametrize("nb", [0, 1, 2, 4, 7, 8, 9, 20])
def test_stencil_reclass_on_output_values(nb):
    """A lone Reclass after a stencil, with breaks drawn from the stencil's
    own outputs so that cells fall exactly on them, and a break at +0 or -0
    under a flat patch (slope exactly 0): up to 8 breaks take the select
    chain of the marching kernels' epilogue, more take the table search,
    and both equal the oracle bit for bit on aligned and strided layouts,
    masked or not, host or device operands."""
    w, h = 300, 200
    dem = dem_cells(w, h, 40 + nb)
    dem[50:80, 40:90] = np.float32(1234.5)
    slope = lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10))
    src = host_raster(dem)
    ref = like(src, masked=False)
    run_oracle(slope(), src, [ref])
    vals = np.unique(ref.data[np.isfinite(ref.data)])
    assert vals[0] == 0 and len(vals) > nb
    rng = np.random.default_rng(nb)
    picked = np.sort(rng.choice(vals[vals > 0], max(nb - 1, 0), replace=False))
    zero = np.float32(-0.0) if nb % 2 else np.float32(0.0)
    breaks = np.concatenate([[zero], picked]).astype(np.float32)[:nb]
    values = (rng.standard_normal(nb + 1) * 5).astype(np.float32)
    values[int(rng.integers(nb + 1))] = np.nan
    make = lambda: slope().extend(transfer.reclass_stage(breaks, values))
    for masked, device in itertools.product((False, True), (False, True)):
        for li, lay in enumerate(layouts(w, h, nb, masked)):
            check_case(make(), dem, 1, device, lay, f"nb={nb} masked={masked} device={device} layout={li}")


def _slope_of_square(s, scale, take_atan):
    """The oracle's slope of a squared gradient magnitude s."""
    from oracle import oracle as orc

    m = np.sqrt(np.asarray(s, np.float32))
    t = orc.atan32_array(m) if take_atan else m
    return (t * np.float32(scale)).astype(np.float32)


def _square_thresholds(breaks, scale, take_atan):
    """Per break, the least non-negative float s whose slope reaches it
    (bisection over the floats in order with the oracle's arithmetic), or
    None when no s does."""
    out = []
    for b in np.asarray(breaks, np.float32):
        lo, hi = 0, 0x7F800000  # bit patterns of +0 and +Inf
        f = lambda u: _slope_of_square(np.array([u], np.uint32).view(np.float32), scale, take_atan)[0]
        if f(hi) < b:
            out.append(None)
            continue
        if f(lo) >= b:
            out.append(np.float32(0))
            continue
        while hi - lo > 1:
            m = (lo + hi) // 2
            if f(m) >= b:
                hi = m
            else:
                lo = m
        out.append(np.array([hi], np.uint32).view(np.float32)[0])
    return out


@pytest.mark.parametrize("units", [0, 1, 2])
def test_slope_class_at_square_thresholds(units):
    """A Slope followed by a Reclass (and the folded Slope -> Lookup ->
    Reclass) runs on the squared gradient magnitude against thresholds the
    host derives; on planes whose squared magnitude lies within a few
    hundred float steps of every class threshold, on both sides of it, the
    device equals the oracle's Slope -> Lookup -> Reclass bit for bit."""
    cs = 10.0
    opts = terrain.SlopeOptions(CellSize=cs, Units=units)
    scale = {0: np.float32(180 / np.pi), 1: np.float32(100), 2: np.float32(1)}[units]
    take_atan = units != 1
    # class breaks in the slope's own unit: the bench's pipeline fold for
    # degrees, spread values for the other units
    breaks = {0: [3.4, 7.9, 15.2, 27.0], 1: [2.0, 9.5, 40.0, 150.0], 2: [0.05, 0.2, 0.6, 1.2]}[units]
    values = [1, 2, 3, 4, 5]
    ts = [t for t in _square_thresholds(breaks, scale, take_atan) if t is not None and t > 0]
    assert len(ts) == len(breaks)
    rng = np.random.default_rng(units)
    bands = []
    for t in ts:
        g = np.sqrt(np.float64(t))
        for phi in (0.0, 0.4, 1.1, 2.9):
            ax, ay = cs * g * np.cos(phi), cs * g * np.sin(phi)
            x0, y0, base = rng.uniform(0, 500), rng.uniform(0, 500), rng.uniform(500, 2500)
            yy, xx = np.mgrid[0:5, 0:256]
            bands.append((base + ax * (xx + x0) + ay * (yy + y0)).astype(np.float32))
    dem = np.concatenate(bands, axis=0)
    h, w = dem.shape
    src = host_raster(dem)
    slope_only = like(src, masked=False)
    run_oracle(terrain.slope_stage(opts), src, [slope_only])
    sl = slope_only.numpy()
    for j, b in enumerate(breaks):
        # the interior rows of the break's four planes
        rows = [j * 20 + p * 5 + k for p in range(4) for k in (1, 2, 3)]
        band = sl[rows][:, 1:-1]
        assert (band < np.float32(b)).any() and (band >= np.float32(b)).any(), f"break {b} not straddled"
    make = lambda: terrain.slope_stage(opts).extend(transfer.reclass_stage(breaks, values))
    make_pipe = lambda: terrain.slope_stage(opts).extend(transfer.lookup_stage([0, 1e6], [0, 1e6])).extend(
        transfer.reclass_stage(breaks, values))
    for mk in (make, make_pipe):
        for device in (False, True):
            lay = dict(src=dict(stride=None, offset=0, valid=None), dst=dict(stride=None, offset=0, masked=False))
            check_case(mk(), dem, 1, device, lay, f"units={units} device={device}")


def test_pipeline_slope_lookup_reclass():
    """The fused Slope -> Lookup -> Reclass pass equals the oracle's three
    stages, which equal three separate calls (internal/exec/pipeline.go)."""
    def stages():
        return (terrain.slope_stage(terrain.SlopeOptions(CellSize=10))
                .extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS))
                .extend(transfer.reclass_stage(BREAKS, VALUES)))

    run_matrix(stages, dem_cells)


def test_pipeline_equals_separate_calls():
    w, h = 200, 77
    cells = dem_cells(w, h, 9)
    valid = synth.block_mask(w, h, 9, 0.05)
    src = host_raster(cells, valid)
    fused = like(src)
    engine.process(terrain.slope_stage(terrain.SlopeOptions(CellSize=10))
                   .extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS))
                   .extend(transfer.reclass_stage(BREAKS, VALUES)), [fused], [src])
    a, b, c = like(src), like(src), like(src)
    terrain.Slope(a, src, terrain.SlopeOptions(CellSize=10))
    transfer.Lookup(b, a, SLOPE_XS, SLOPE_YS)
    transfer.Reclass(c, b, BREAKS, VALUES)
    assert_same_raster(fused, c, "pipeline vs separate")


def test_in_place_pointwise():
    """A pointwise op may run in place (dst is src), as transfer allows."""
    w, h = 100, 30
    cells = poison(synth.normal_trend(w, h, 3) * 10, 3)
    src = host_raster(cells, synth.cell_mask(w, h, 3))
    want = like(src)
    run_oracle(transfer.reclass_stage(BREAKS, VALUES), src, [want])
    engine.process(transfer.reclass_stage(BREAKS, VALUES), [src], [src])
    assert_same_raster(src, want, "in place")


def test_edges_are_nan_and_invalid():
    w, h = 40, 30
    src = host_raster(dem_cells(w, h, 4), np.ones((h, w), bool))
    for r in (1, 4, 8):
        dst = like(src)
        focal.Mean(dst, src, focal.BoxOptions(Radius=r))
        a = dst.numpy()
        v = dst.valid_numpy()
        ring = np.ones((h, w), bool)
        ring[r:h - r, r:w - r] = False
        assert np.isnan(a[ring]).all() and not v[ring].any()
        assert v[~ring].all()


def test_window_smaller_than_radius_is_all_edge():
    for w, h, r in ((5, 40, 3), (40, 2, 1), (16, 16, 8)):
        src = host_raster(focal_cells(w, h, 1), np.ones((h, w), bool))
        dst = like(src)
        focal.Max(dst, src, focal.BoxOptions(Radius=r))
        assert np.isnan(dst.numpy()).all() and not dst.valid_numpy().any()


def test_tiled_options_give_the_same_bits():
    """Tiled entry points write the same bits for every engine.Options
    (the reference's TestTilesAndWorkers rule)."""
    w, h = 300, 200
    src = host_raster(dem_cells(w, h, 5), synth.cell_mask(w, h, 5))
    want = like(src)
    terrain.Slope(want, src, terrain.SlopeOptions(CellSize=30))
    for tw, th, workers in ((1, 1, 1), (7, 64, 2), (256, 3, 3), (0, 0, 0), (1 << 20, 1 << 20, 8)):
        got = like(src)
        st = engine.Stats()
        err = terrain.SlopeTiled(engine.Background(), got, src, terrain.SlopeOptions(CellSize=30),
                                 engine.Options(TileWidth=tw, TileHeight=th, Workers=workers, Stats=st))
        assert err is None
        assert_same_raster(got, want, f"tiled {tw}x{th}")
        assert st.Cells == w * h and st.Ideal == w * h * 8 and st.KernelWritten == w * h * 4
        assert st.KernelRead >= w * h * 4


@pytest.mark.parametrize("tile", [(1, 1), (7, 5), (64, 64), (300, 13), (0, 0), (1000, 1000)])
def test_chunked_equals_plain(tile):
    """Chunked through memory sources and sinks writes the plain call's bits
    (internal/exec/chunked_test.go:162-200), for several tile shapes."""
    w, h = 150, 90
    src = host_raster(dem_cells(w, h, 6), synth.block_mask(w, h, 6, 0.05))
    for name, mk in (("slope", lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=30))),
                     ("tpi r3", lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2, Radius=3))),
                     ("max r4", lambda: focal.box_stage(focal.BoxOptions(Radius=4), engine._lib.OP_MAX))):
        want = like(src)
        engine.process(mk(), [want], [src])
        got = like(src)
        st = engine.Stats()
        err = engine.process_chunked(mk(), [engine.MemorySink(got)], [engine.MemorySource(src)],
                                     engine.Options(TileWidth=tile[0], TileHeight=tile[1], Stats=st))
        assert err is None
        assert_same_raster(got, want, f"chunked {name} {tile}")
        assert st.Cells == w * h and st.SinkWritten == w * h * 4
        tw = tile[0] if tile[0] else w
        th = tile[1] if tile[1] else h
        assert st.Tiles == -(-w // min(tw, w)) * -(-h // min(th, h))


def test_chunked_gradient_two_sinks():
    w, h = 77, 51
    src = host_raster(dem_cells(w, h, 8), synth.cell_mask(w, h, 8))
    want = [like(src), like(src)]
    terrain.Gradient(want[0], want[1], src, terrain.GradientOptions(CellSize=30))
    got = [like(src), like(src)]
    err = terrain.GradientChunked(engine.Background(), engine.MemorySink(got[0]), engine.MemorySink(got[1]),
                                  engine.MemorySource(src), terrain.GradientOptions(CellSize=30),
                                  engine.Options(TileWidth=20, TileHeight=16))
    assert err is None
    assert_same_raster(got[0], want[0], "dx")
    assert_same_raster(got[1], want[1], "dy")


def test_slope_c1_size_against_oracle():
    """Slope on the 2048 x 2048 workload (CellSize 30, 2% NoData in 8x8
    blocks) equals the oracle on every cell."""
    w = h = 2048
    seed = 0x5EED0001
    src = host_raster(synth.fbm_dem(w, h, seed), synth.block_mask(w, h, seed))
    want, got = like(src), like(src)
    run_oracle(terrain.slope_stage(terrain.SlopeOptions(CellSize=30)), src, [want], nthreads=8)
    terrain.Slope(got, src, terrain.SlopeOptions(CellSize=30))
    assert_same_raster(got, want, "slope 2048")


FOCAL_LARGE = {
    "mean_r8": lambda: focal.box_stage(focal.BoxOptions(Radius=8), engine._lib.OP_MEAN),
    "min_r3": lambda: focal.box_stage(focal.BoxOptions(Radius=3), engine._lib.OP_MIN),
    "max_r5": lambda: focal.box_stage(focal.BoxOptions(Radius=5), engine._lib.OP_MAX),
    "gaussian_r8": lambda: focal.separable_stage(focal.SeparableOptions(8, focal.Gaussian(8, 2.5),
                                                                        synth.uniform_weights(17, 9))),
    "roughness_r6": lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=3, Radius=6)),
    "correlate_r8": lambda: focal.weights_stage(focal.WeightsOptions(8, synth.uniform_weights(289, 3)), False),
    "convolve_r2": lambda: focal.weights_stage(focal.WeightsOptions(2, synth.uniform_weights(25, 4)), True),
    "riley_r4": lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=0, Radius=4)),
    "wilson_r7": lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=1, Radius=7)),
    "tpi_r2": lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2, Radius=2)),
    "mean_r8_reclass": lambda: focal.box_stage(focal.BoxOptions(Radius=8), engine._lib.OP_MEAN).extend(
        transfer.reclass_stage([-0.5, 0.0, 0.5], [1, 2, 3, 4])),
}


@pytest.mark.parametrize("name", sorted(FOCAL_LARGE))
def test_focal_large_against_oracle(name):
    """The focal ops at radius 2..8 over a raster wide and tall enough for
    many column blocks, bands and tiles (5% NoData cells), and over a
    window view of it at an offset, equal the oracle on every cell and bit."""
    w, h = 2052, 700
    seed = 0x5EED0003
    src = host_raster(poison(synth.normal_trend(w, h, seed), seed, 0.001), synth.cell_mask(w, h, seed, 0.05))
    want, got = like(src), like(src)
    run_oracle(FOCAL_LARGE[name](), src, [want], nthreads=8)
    dsrc, dgot = to_device(src), to_device(got)
    assert engine.process(FOCAL_LARGE[name](), [dgot], [dsrc]) is None
    assert_same_raster(to_host(dgot), want, name)
    # a window view: its own raster, with the parent's stride and bit offsets
    win = dsrc.Window(36, 21, 1500, 611)
    wwant = like(to_host(win))
    run_oracle(FOCAL_LARGE[name](), to_host(win), [wwant], nthreads=8)
    wgot = to_device(like(to_host(win)))
    assert engine.process(FOCAL_LARGE[name](), [wgot], [win]) is None
    assert_same_raster(to_host(wgot), wwant, name + " window")


def test_features_equal_separate_calls():
    """terrain.Features (terrain/features.go): every output equals its op run
    alone, with mixed radii (each output its own edge ring), host and device."""
    w, h = 203, 71
    cells = dem_cells(w, h, 12)
    src = host_raster(cells, synth.block_mask(w, h, 12, 0.05))
    ops = [terrain.SlopeOptions(CellSize=10), terrain.AspectOptions(CellSize=10),
           terrain.HillshadeOptions(CellSize=10), terrain.CurvatureOptions(CellSize=10, Type=1),
           terrain.RuggednessOptions(Type=terrain.RuggednessTPI, Radius=3),
           terrain.RuggednessOptions(Type=terrain.RuggednessRoughness)]
    singles = {terrain.SlopeOptions: terrain.Slope, terrain.AspectOptions: terrain.Aspect,
               terrain.HillshadeOptions: terrain.Hillshade, terrain.CurvatureOptions: terrain.Curvature,
               terrain.RuggednessOptions: terrain.Ruggedness}
    for device in (False, True):
        s = to_device(src) if device else src
        outs = [to_device(like(src)) if device else like(src) for _ in ops]
        terrain.Features([terrain.Feature(op, d) for op, d in zip(ops, outs)], s)
        for op, got in zip(ops, outs):
            want = like(src)
            singles[type(op)](want, src, op)
            assert_same_raster(to_host(got), want, f"features {type(op).__name__} device={device}")


def _fused_feature_set():
    """Every radius-1 op and kind, with Reclass epilogues (folded on the
    squared magnitude for Slope), and one radius-3 op: the memory-bound
    ones run in the fused pass, the others as their own launches."""
    o = dict(CellSize=10)
    return [
        terrain.gradient_stage(terrain.GradientOptions(CellSize=10, CellSizeY=12)),
        terrain.slope_stage(terrain.SlopeOptions(**o)),
        terrain.slope_stage(terrain.SlopeOptions(CellSize=3, Units=terrain.SlopePercent)),
        terrain.aspect_stage(terrain.AspectOptions(**o)),
        terrain.aspect_stage(terrain.AspectOptions(CellSize=5, ZeroForFlat=True, Trigonometric=True)),
        terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10, Azimuth=200, Altitude=30)),
        terrain.curvature_stage(terrain.CurvatureOptions(Type=0, **o)),
        terrain.curvature_stage(terrain.CurvatureOptions(Type=1, **o)),
        terrain.curvature_stage(terrain.CurvatureOptions(Type=2, **o)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=0)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=1)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=3)),
        terrain.slope_stage(terrain.SlopeOptions(**o)).extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS)).extend(
            transfer.reclass_stage(BREAKS, VALUES)),
        terrain.slope_stage(terrain.SlopeOptions(CellSize=2, Units=terrain.SlopePercent)).extend(
            transfer.reclass_stage([5, 15, 60], [1, 2, 3, 4])),
        terrain.aspect_stage(terrain.AspectOptions(**o)).extend(transfer.reclass_stage([90, 180, 270], [1, 2, 3, 4])),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2, Radius=3)),
    ]


@pytest.mark.parametrize("w,h", [(256, 70), (516, 37), (1028, 9)])
def test_fused_features_equal_separate_calls_and_oracle(w, h):
    """One Features call over every radius-1 op (the memory-bound ones in
    the fused multi-output pass) writes each output's own bits and validity:
    the same as the op run alone and as the oracle, masked and unmasked,
    host and device operands, compact and strided outputs with bit offsets."""
    cells = dem_cells(w, h, w + h)
    for masked, device, strided in itertools.product((False, True), (False, True), (False, True)):
        src = host_raster(cells, synth.block_mask(w, h, w, 0.05) if masked else None)
        feats = _fused_feature_set()
        nouts = [2 if f.stages[0].op == engine._lib.OP_GRADIENT else 1 for f in feats]
        st, off = (w + 8, 40) if strided else (None, 0)
        outs = [like(src, st, off) for _ in range(sum(nouts))]
        before = [Float32Raster(np.array(g.data), g.width, g.height, g.stride,
                                None if g.valid is None else np.array(g.valid), g.valid_offset) for g in outs]
        s_ = to_device(src) if device else src
        o_ = [to_device(x) for x in outs] if device else outs
        assert engine.process_features(feats, o_, s_) is None
        got = [to_host(x) for x in o_] if device else outs
        k = 0
        for f, n in zip(_fused_feature_set(), nouts):
            alone = [like(src, st, off) for _ in range(n)]
            assert engine.process(f, alone, [src]) is None
            want = [like(src, st, off) for _ in range(n)]
            run_oracle(f, src, want)
            for i in range(n):
                what = f"{w}x{h} masked={masked} device={device} strided={strided} feature op {f.stages[0].op} out{i}"
                assert_same_raster(got[k + i], alone[i], what + " vs alone")
                assert_same_raster(got[k + i], want[i], what + " vs oracle")
                assert_padding_untouched(before[k + i], got[k + i], what)
            k += n


CARRIERS = {
    "slope_deg": lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10)),
    "slope_rad_reclass": lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=3, Units=terrain.SlopeRadians)).extend(
        transfer.reclass_stage([0.1, 0.5, 1.0], [1, 2, 3, 4])),
    "aspect_trig": lambda: terrain.aspect_stage(terrain.AspectOptions(CellSize=5, Trigonometric=True)),
    "hillshade": lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10, Azimuth=200, Altitude=30)),
    "curv_profile": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=0)),
    "curv_plan": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=1)),
    "curv_mean_reclass": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=2)).extend(
        transfer.reclass_stage([-0.01, 0, 0.01], [1, 2, 3, 4])),
    "tri_riley": lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=0)),
}


@pytest.mark.parametrize("name", sorted(CARRIERS))
def test_fused_pass_carried_by_each_product(name):
    """The memory-bound features carried by one arithmetic-bound product
    in the fused pass: every output equals its op run alone and the oracle,
    masked and unmasked, compact and strided outputs."""
    w, h = 388, 53
    cells = dem_cells(w, h, len(name))
    for masked, strided in itertools.product((False, True), (False, True)):
        src = host_raster(cells, synth.block_mask(w, h, w, 0.05) if masked else None)
        feats = lambda: [terrain.gradient_stage(terrain.GradientOptions(CellSize=10)), CARRIERS[name](),
                         terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2)),
                         terrain.ruggedness_stage(terrain.RuggednessOptions(Type=3))]
        nouts = [2, 1, 1, 1]
        st, off = (w + 8, 40) if strided else (None, 0)
        outs = [like(src, st, off) for _ in range(sum(nouts))]
        assert engine.process_features(feats(), outs, src) is None
        k = 0
        for f, n in zip(feats(), nouts):
            alone = [like(src, st, off) for _ in range(n)]
            assert engine.process(f, alone, [src]) is None
            want = [like(src, st, off) for _ in range(n)]
            run_oracle(f, src, want)
            for i in range(n):
                what = f"{name} masked={masked} strided={strided} op {f.stages[0].op} out{i}"
                assert_same_raster(outs[k + i], alone[i], what + " vs alone")
                assert_same_raster(outs[k + i], want[i], what + " vs oracle")
            k += n


def test_features_over_many_units_two_streams():
    """A Features call on a raster of thousands of strip units, the ops that
    run as their own launches alternating over two streams, twice on the
    same context: every output equals its op run alone."""
    w, h = 1032, 3001
    src = to_device(host_raster(dem_cells(w, h, 77), synth.block_mask(w, h, 77, 0.03)))
    feats = lambda: [terrain.gradient_stage(terrain.GradientOptions(CellSize=10)),
                     terrain.aspect_stage(terrain.AspectOptions(CellSize=10)),
                     terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2)),
                     terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=1)),
                     terrain.ruggedness_stage(terrain.RuggednessOptions(Type=3))]
    nouts = [2, 1, 1, 1, 1]
    outs = [to_device(like(to_host(src))) for _ in range(sum(nouts))]
    for _ in range(2):  # the second call reuses the context's streams
        assert engine.process_features(feats(), outs, src) is None
    k = 0
    for f, n in zip(feats(), nouts):
        alone = [to_device(like(to_host(src))) for _ in range(n)]
        assert engine.process(f, alone, [src]) is None
        for i in range(n):
            assert_same_raster(to_host(outs[k + i]), to_host(alone[i]), f"op {f.stages[0].op} out{i}")
        k += n


def test_surface_equals_separate_calls():
    w, h = 128, 40
    src = host_raster(dem_cells(w, h, 13), synth.cell_mask(w, h, 13))
    o = terrain.SurfaceOptions(CellSize=5, Units=terrain.SlopePercent, Azimuth=200, Altitude=30)
    out = terrain.SurfaceOutputs(Dx=like(src), Dy=like(src), Slope=like(src), Aspect=like(src),
                                 Hillshade=like(src))
    terrain.Surface(out, src, o)
    dx, dy, sl, asp, hs = like(src), like(src), like(src), like(src), like(src)
    terrain.Gradient(dx, dy, src, terrain.GradientOptions(CellSize=5))
    terrain.Slope(sl, src, terrain.SlopeOptions(CellSize=5, Units=terrain.SlopePercent))
    terrain.Aspect(asp, src, terrain.AspectOptions(CellSize=5))
    terrain.Hillshade(hs, src, terrain.HillshadeOptions(CellSize=5, Azimuth=200, Altitude=30))
    for got, want, n in ((out.Dx, dx, "dx"), (out.Dy, dy, "dy"), (out.Slope, sl, "slope"),
                         (out.Aspect, asp, "aspect"), (out.Hillshade, hs, "hillshade")):
        assert_same_raster(got, want, f"surface {n}")
    only = terrain.SurfaceOutputs(Dy=like(src))
    terrain.Surface(only, src, o)
    assert_same_raster(only.Dy, dy, "surface dy alone")


def test_graph_run_equals_engine():
    from strata_b200 import graph

    w, h = 96, 50
    src = host_raster(dem_cells(w, h, 14), synth.block_mask(w, h, 14, 0.05))
    g = graph.New()
    dem = g.Input("dem")
    g.Output("class", graph.Reclass(graph.Lookup(graph.Slope(dem, terrain.SlopeOptions(CellSize=10)),
                                                 SLOPE_XS, SLOPE_YS), BREAKS, VALUES))
    out = like(src)
    assert g.Plan().Run(engine.Background(), {"dem": src}, {"class": out}) is None
    want = like(src)
    run_oracle(terrain.slope_stage(terrain.SlopeOptions(CellSize=10)).extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS))
               .extend(transfer.reclass_stage(BREAKS, VALUES)), src, [want])
    assert_same_raster(out, want, "graph")


def test_cancel_before_start_returns_canceled():
    w, h = 64, 64
    src = host_raster(dem_cells(w, h, 15))
    dst = like(src)
    ctx = engine.Context()
    ctx.cancel()
    err = terrain.SlopeTiled(ctx, dst, src, terrain.SlopeOptions(CellSize=1), engine.Options())
    assert isinstance(err, engine.Canceled)


def test_chunked_source_error_is_returned():
    """A failing source ends the call with its error, wrapped with the
    operand and position (internal/exec/chunked.go:379-393), and the sink
    holds only whole tiles in plan order before it."""
    w, h = 64, 48
    src = host_raster(dem_cells(w, h, 16))

    class Failing(engine.MemorySource):
        def ReadWindow(self, dst, x, y):
            if y > 20:
                return IOError("disk on fire")
            return super().ReadWindow(dst, x, y)

    got = like(src)
    err = terrain.SlopeChunked(engine.Background(), engine.MemorySink(got), Failing(src),
                               terrain.SlopeOptions(CellSize=1), engine.Options(TileWidth=64, TileHeight=16))
    assert isinstance(err, engine.SourceSinkError) and "disk on fire" in str(err) and "src[0]" in str(err)
    want = like(src)
    terrain.Slope(want, src, terrain.SlopeOptions(CellSize=1))
    from helpers import same_bits

    assert same_bits(got.numpy()[:16], want.numpy()[:16]).all()


# ---------------------------------------------------------------------------
# HeatLoad and Orientation (Horn's gradient) and Wood's quadratic fit
# (FitRadius 1..8) for every product.

HEAT_ORIENT = {
    "heat_eq1": lambda: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=10, Latitude=40)),
    "heat_eq2_rad_south": lambda: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=5, CellSizeY=7,
                                                                                  Latitude=-35, Equation=1,
                                                                                  Radiation=True)),
    "heat_eq3": lambda: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=30, Latitude=52.5, Equation=2)),
    "north": lambda: terrain.orientation_stage(terrain.OrientationOptions(CellSize=10)),
    "east_unweighted": lambda: terrain.orientation_stage(terrain.OrientationOptions(CellSize=3, ZFactor=2,
                                                                                    Component=terrain.Eastness,
                                                                                    Unweighted=True)),
}


@pytest.mark.parametrize("name", sorted(HEAT_ORIENT))
def test_heatload_orientation(name):
    run_matrix(HEAT_ORIENT[name], dem_cells, shapes=SHAPES[:9])


def test_heatload_linear_within_one_ulp():
    """With Linear, Equations 1 and 2 take exp of the regression: CUDA's exp
    and the C library's (and Go's math.Exp) agree to a float64 ulp, so the
    float32 result may move by one ulp where the sum sits at a rounding
    boundary; every other cell and every validity bit is exact."""
    w, h = 257, 131
    cells = dem_cells(w, h, 77)
    src = host_raster(cells, synth.cell_mask(w, h, 77, 0.03))
    st = lambda: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=10, Latitude=44, Linear=True))
    want, got = like(src), like(src)
    run_oracle(st(), src, [want])
    assert engine.process(st(), [got], [src]) is None
    g, wv = got.numpy(), want.numpy()
    both_nan = np.isnan(g) & np.isnan(wv)
    ulps = np.abs(g.view(np.int32).astype(np.int64) - wv.view(np.int32).astype(np.int64))
    assert (both_nan | (ulps <= 1)).all()
    assert (got.valid_numpy() == want.valid_numpy()).all()


FIT_PRODUCTS = {
    "gradient": (lambda r: terrain.gradient_stage(terrain.GradientOptions(CellSize=10, CellSizeY=12, FitRadius=r)), 2),
    "slope_deg": (lambda r: terrain.slope_stage(terrain.SlopeOptions(CellSize=10, FitRadius=r)), 1),
    "slope_pct": (lambda r: terrain.slope_stage(terrain.SlopeOptions(CellSize=10, Units=terrain.SlopePercent,
                                                                     FitRadius=r)), 1),
    "aspect": (lambda r: terrain.aspect_stage(terrain.AspectOptions(CellSize=10, Trigonometric=True, FitRadius=r)), 1),
    "hillshade": (lambda r: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10, Azimuth=120, FitRadius=r)),
                  1),
    "heatload": (lambda r: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=10, Latitude=47, Equation=2,
                                                                          FitRadius=r)), 1),
    "orientation": (lambda r: terrain.orientation_stage(terrain.OrientationOptions(CellSize=10, FitRadius=r)), 1),
    "curv_profile": (lambda r: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=0, FitRadius=r)), 1),
    "curv_plan": (lambda r: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=1, FitRadius=r)), 1),
    "curv_mean": (lambda r: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=4, CellSizeY=6, ZFactor=2,
                                                                             Type=2, FitRadius=r)), 1),
    "slope_classes": (lambda r: terrain.slope_stage(terrain.SlopeOptions(CellSize=10, FitRadius=r)).extend(
        transfer.lookup_stage(SLOPE_XS, SLOPE_YS)).extend(transfer.reclass_stage(BREAKS, VALUES)), 1),
}


@pytest.mark.parametrize("name", sorted(FIT_PRODUCTS))
@pytest.mark.parametrize("r", [1, 2, 5, 8])
def test_wood_fit_products(name, r):
    """Wood's fit (terrain/fit.go) on the device (raw sums as separable
    correlations, then the finishing pass) against the oracle's fit, cell
    for cell and bit for bit, over small and odd shapes and layouts."""
    make, nout = FIT_PRODUCTS[name]
    run_matrix(lambda: make(r), dem_cells, nout=nout, shapes=SMALL_SHAPES, seed=r)


def test_fit_surface_and_features_equal_standalone():
    """TestFitSurfaceIsTheStandaloneProducts (terrain/fit_test.go:134-204):
    a Features call with FitRadius set writes what each product alone does."""
    w, h = 96, 40
    src = host_raster(dem_cells(w, h, 21), synth.block_mask(w, h, 21, 0.05))
    ops = [terrain.SlopeOptions(CellSize=10, FitRadius=3), terrain.AspectOptions(CellSize=10, FitRadius=3),
           terrain.HeatLoadOptions(CellSize=10, Latitude=30, FitRadius=2),
           terrain.OrientationOptions(CellSize=10, Component=terrain.Eastness),
           terrain.CurvatureOptions(CellSize=10, Type=2, FitRadius=4)]
    singles = {terrain.SlopeOptions: terrain.Slope, terrain.AspectOptions: terrain.Aspect,
               terrain.HeatLoadOptions: terrain.HeatLoad, terrain.OrientationOptions: terrain.Orientation,
               terrain.CurvatureOptions: terrain.Curvature}
    outs = [like(src) for _ in ops]
    terrain.Features([terrain.Feature(op, d) for op, d in zip(ops, outs)], src)
    for op, got in zip(ops, outs):
        want = like(src)
        singles[type(op)](want, src, op)
        assert_same_raster(got, want, f"features {type(op).__name__}")


@pytest.mark.parametrize("r", [1, 3, 8])
def test_fit_chunked_equals_plain(r):
    """Wood's fit through the chunked form (tiles with the fit's halo, the
    sums in context scratch per tile) writes the plain call's bits."""
    w, h = 517, 203
    src = host_raster(dem_cells(w, h, 5 + r), synth.block_mask(w, h, r, 0.03))
    st = lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=2, FitRadius=r))
    plain, chunked = like(src), like(src)
    assert engine.process(st(), [plain], [src]) is None
    assert engine.process_chunked(st(), [engine.MemorySink(chunked)], [engine.MemorySource(src)],
                                  engine.Options(TileWidth=200, TileHeight=64)) is None
    assert_same_raster(chunked, plain, f"fit r={r} chunked")


def test_fit_has_no_batch_form():
    from strata_b200 import batch
    from strata_b200.raster import NotSupported

    w, h = 40, 30
    src = to_device(host_raster(dem_cells(w, h, 5)))
    with pytest.raises(NotSupported):
        batch.Batch([batch.Item(terrain.slope_stage(terrain.SlopeOptions(CellSize=1, FitRadius=2)), src,
                                [to_device(like(to_host(src)))])])


def test_heatload_orientation_in_a_batch():
    """HeatLoad and Orientation run in the batched form: every raster equals
    its plain call."""
    from strata_b200 import batch

    rng = np.random.default_rng(3)
    items, outs, wants = [], [], []
    makers = [lambda: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=10, Latitude=40, Equation=1)),
              lambda: terrain.heatload_stage(terrain.HeatLoadOptions(CellSize=30, Latitude=-20, Linear=True)),
              lambda: terrain.orientation_stage(terrain.OrientationOptions(CellSize=10)),
              lambda: terrain.orientation_stage(terrain.OrientationOptions(CellSize=5, Component=terrain.Eastness,
                                                                           Unweighted=True))]
    for i in range(8):
        w, h = int(rng.integers(30, 600)), int(rng.integers(10, 300))
        hsrc = host_raster(dem_cells(w, h, i), synth.block_mask(w, h, i, 0.03))
        st = makers[i % 4]
        want = like(hsrc)
        assert engine.process(st(), [want], [hsrc]) is None
        out = to_device(like(hsrc))
        items.append(batch.Item(st(), to_device(hsrc), [out]))
        outs.append(out)
        wants.append(want)
    b = batch.Batch(items)
    b.run()
    b.close()
    for i, (o, w_) in enumerate(zip(outs, wants)):
        assert_same_raster(to_host(o), w_, f"batch item {i}")
