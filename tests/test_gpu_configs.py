"""Parity at the benchmarked configurations' own widths and offsets, not
only at the engine matrix's small shapes: every op of the 16384-wide
terrain set, and the 8192-wide focal set, on row bands with their masks,
against the oracle cell for cell (rastertest.SameFloat) and bit for bit;
and served windows deep inside a device-resident mosaic of more than 2^31
cells (byte offsets past 2^33, bit offsets past 2^31), against
strata_process on the same window view."""
from __future__ import annotations

import pytest

from helpers import assert_same_raster, host_raster, like, run_oracle, to_device, to_host
from strata_b200 import engine, focal, serve, synth, terrain, transfer
from strata_b200.raster import Float32Raster

pytestmark = pytest.mark.gpu

SLOPE_XS, SLOPE_YS = [0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5]
BREAKS, VALUES = [1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5]


def _terrain_set(cs):
    o = dict(CellSize=cs)
    return [
        terrain.gradient_stage(terrain.GradientOptions(**o)),
        terrain.slope_stage(terrain.SlopeOptions(**o)),
        terrain.aspect_stage(terrain.AspectOptions(**o)),
        terrain.hillshade_stage(terrain.HillshadeOptions(Azimuth=315, Altitude=45, ZFactor=1, **o)),
        terrain.curvature_stage(terrain.CurvatureOptions(Type=0, **o)),
        terrain.curvature_stage(terrain.CurvatureOptions(Type=1, **o)),
        terrain.curvature_stage(terrain.CurvatureOptions(Type=2, **o)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=0, Radius=1)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2, Radius=1)),
        terrain.ruggedness_stage(terrain.RuggednessOptions(Type=3, Radius=1)),
        terrain.slope_stage(terrain.SlopeOptions(**o)).extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS)).extend(
            transfer.reclass_stage(BREAKS, VALUES)),
    ]


def test_terrain_set_16384_wide_band():
    """The terrain set's workload width (16384, CellSize 10, 2% NoData in 8x8
    blocks), a 48-row band, through one Features call (the fused pass and
    the separate launches) on device operands."""
    w, h = 16384, 48
    cells = synth.fbm_dem(w, h, 0x5EED0002)
    valid = synth.block_mask(w, h, 0x5EED0002, 0.02)
    src = host_raster(cells, valid)
    feats = _terrain_set(10)
    nouts = [2 if f.stages[0].op == engine._lib.OP_GRADIENT else 1 for f in feats]
    outs = [to_device(like(src)) for _ in range(sum(nouts))]
    assert engine.process_features(feats, outs, to_device(src)) is None
    k = 0
    for f, n in zip(_terrain_set(10), nouts):
        want = [like(src) for _ in range(n)]
        run_oracle(f, src, want, nthreads=8)
        for i in range(n):
            assert_same_raster(to_host(outs[k + i]), want[i], f"op {f.stages[0].op} out{i}")
        k += n


@pytest.mark.parametrize("r", [3, 8])
def test_focal_set_8192_wide_band(r):
    """The focal workload's width (8192, N(0,1) plus trend, 5% random NoData)
    at radius 3 and 8: Correlate, Gaussian, Mean, Min, Max."""
    w, h = 8192, 2 * r + 40
    cells = synth.normal_trend(w, h, 0x5EED0003)
    src = host_raster(cells, synth.cell_mask(w, h, 0x5EED0003, 0.05))
    wts = synth.uniform_weights((2 * r + 1) ** 2, 0x5EED0003 + r)
    g = focal.Gaussian(r, 2.5)
    ops = [focal.weights_stage(focal.WeightsOptions(r, wts), False),
           focal.separable_stage(focal.SeparableOptions(r, g, g))] + \
        [focal.box_stage(focal.BoxOptions(r), op) for op in (engine._lib.OP_MEAN, engine._lib.OP_MIN,
                                                              engine._lib.OP_MAX)]
    dsrc = to_device(src)
    for st in ops:
        got = to_device(like(src))
        assert engine.process(st, [got], [dsrc]) is None
        want = like(src)
        run_oracle(st, src, [want], nthreads=8)
        assert_same_raster(to_host(got), want, f"op {st.stages[0].op} r={r}")


def test_served_window_deep_in_a_mosaic_past_2e31_cells():
    """A 47000 x 47000 mosaic (8.8 GB of cells, a 276 MB mask) resident on
    the device; windows at its far corner and across its last rows (byte
    offsets past 2^33, bit offsets past 2^31) are served and equal
    strata_process on the same window view bit for bit."""
    import torch

    n = 47000
    assert n * n > 1 << 31
    g = torch.Generator(device="cuda").manual_seed(7)
    cells = torch.empty(n * n, dtype=torch.float32, device="cuda")
    for y0 in range(0, n, 2000):  # a gentle surface with noise, a band at a time
        ys = torch.arange(y0, min(n, y0 + 2000), device="cuda", dtype=torch.float32)[:, None]
        xs = torch.arange(n, device="cuda", dtype=torch.float32)[None, :]
        band = 500 + 0.01 * xs + 0.02 * ys + torch.randn((ys.shape[0], n), device="cuda", generator=g)
        cells[y0 * n:(y0 + ys.shape[0]) * n] = band.reshape(-1)
    words = (n * n + 63) // 64
    valid = torch.randint(-(1 << 62), 1 << 62, (words,), device="cuda", dtype=torch.int64, generator=g)
    valid |= torch.randint(-(1 << 62), 1 << 62, (words,), device="cuda", dtype=torch.int64, generator=g)
    mosaic = Float32Raster(cells, n, n, n, valid, 0)
    wins = [(n - 700, n - 500, 700, 500), (n - 4096, n - 300, 4096, 300), (n - 257, n - 1030, 257, 1030)]
    ops = [terrain.slope_stage(terrain.SlopeOptions(CellSize=30)),
           focal.box_stage(focal.BoxOptions(Radius=5), engine._lib.OP_MEAN),
           terrain.ruggedness_stage(terrain.RuggednessOptions(Type=terrain.RuggednessTPI))]
    srv = serve.Server(mosaic, budget_bytes=8 << 30, streams=2, max_batch=8)
    try:
        for x, y, w, h in wins:
            assert y * n + x > 1 << 31
            for st in ops:
                t = srv.submit(st, x, y, w, h)
                res = srv.wait(t)
                win = mosaic.Window(x, y, w, h)
                alone = Float32Raster(torch.empty(w * h, dtype=torch.float32, device="cuda"), w, h, w,
                                      torch.zeros((w * h + 63) // 64, dtype=torch.int64, device="cuda"), 0)
                assert engine.process(st, [alone], [win]) is None
                assert_same_raster(to_host(res.copy(0)), to_host(alone), f"window {w}x{h} at ({x}, {y})")
                srv.release(t)
    finally:
        srv.close()
    del cells, valid, mosaic
    torch.cuda.empty_cache()
