"""strata_batch_run_noalloc (descriptors in the library's static device
scratch, no allocation) against strata_batch_create + strata_batch_run on
the same items, through the C ABI. Both run the same batch kernels, so the
tolerance is zero: bit-identical data and validity.

Two calls in a row go on one stream with no wait between them, the second
over different rasters, so the second call's descriptors overwrite the
scratch only after the first call's kernels have read it (stream order)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from helpers import assert_same_raster, host_raster, like, to_device, to_host
from strata_b200 import _lib, engine, focal, synth, terrain, transfer

pytestmark = pytest.mark.gpu


def _stages(rng):
    r = int(rng.integers(1, 9))
    choices = [
        lambda: (terrain.slope_stage(terrain.SlopeOptions(CellSize=float(rng.uniform(1, 90)))), 1),
        lambda: (terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=30)), 1),
        lambda: (terrain.gradient_stage(terrain.GradientOptions(CellSize=30)), 2),
        lambda: (focal.weights_stage(focal.WeightsOptions(r, synth.uniform_weights((2 * r + 1) ** 2, r)), False), 1),
        lambda: (focal.box_stage(focal.BoxOptions(r), _lib.OP_MAX), 1),
        lambda: (terrain.ruggedness_stage(terrain.RuggednessOptions(Type=int(rng.integers(4)), Radius=r)), 1),
        lambda: (terrain.slope_stage(terrain.SlopeOptions(CellSize=10)).extend(
            transfer.reclass_stage([2, 5, 10, 20], [1, 2, 3, 4, 5])), 1),
    ]
    return choices[int(rng.integers(len(choices)))]()


def _set(seed, n):
    """n rasters of mixed sizes, ops, masks and tiles: (stages, src, host src, nout, tile)."""
    rng = np.random.default_rng(seed)
    tiles = [(0, 0), (64, 32), (128, 16), (32, 8)]
    out = []
    for i in range(n):
        w = int(np.exp(rng.uniform(np.log(3), np.log(700))))
        h = int(np.exp(rng.uniform(np.log(3), np.log(700))))
        mask = synth.cell_mask(w, h, seed + i, 0.03) if rng.integers(2) else None
        src = host_raster(synth.fbm_dem(w, h, seed * 100 + i), mask)
        stages, nout = _stages(rng)
        out.append((stages, to_device(src), src, nout, tiles[i % len(tiles)]))
    return out


def _c_items(spec, dsts):
    arr = (_lib.BatchItem * len(spec))()
    keep = []
    for i, (stages, dsrc, _, nout, tile) in enumerate(spec):
        st = stages.c_array()
        keep += [st, stages]
        arr[i].stages = ctypes.cast(st, ctypes.POINTER(_lib.Stage))
        arr[i].nstages = len(stages.stages)
        arr[i].tile_width, arr[i].tile_height = tile
        arr[i].src = engine.c_raster(dsrc)
        for k in range(nout):
            arr[i].dst[k] = engine.c_raster(dsts[i][k])
    return arr, keep


def _outputs(spec):
    return [[to_device(like(src)) for _ in range(nout)] for _, _, src, nout, _ in spec]


def _run_existing(ctx, spec):
    dsts = _outputs(spec)
    arr, _keep = _c_items(spec, dsts)
    L = _lib.lib()
    b = ctypes.c_void_p()
    _lib.check(L.strata_batch_create(ctx, arr, len(spec), ctypes.byref(b)))
    try:
        _lib.check(L.strata_batch_run(b, None, 1))
    finally:
        L.strata_batch_destroy(b)
    return dsts


def test_noalloc_equals_batch_two_calls_in_a_row():
    import torch

    ctx = engine.device_context(0)
    L = _lib.lib()
    specs = [_set(11, 24), _set(12, 40)]
    want = [_run_existing(ctx, s) for s in specs]
    got = [_outputs(s) for s in specs]
    c_items = [_c_items(s, g) for s, g in zip(specs, got)]
    stream = torch.cuda.Stream()
    # back to back on one stream; only the second call waits
    _lib.check(L.strata_batch_run_noalloc(ctx, c_items[0][0], len(specs[0]), stream.cuda_stream, 0))
    _lib.check(L.strata_batch_run_noalloc(ctx, c_items[1][0], len(specs[1]), stream.cuda_stream, 1))
    for c, (spec, g, w) in enumerate(zip(specs, got, want)):
        for i, (stages, _, src, nout, tile) in enumerate(spec):
            for k in range(nout):
                assert_same_raster(to_host(g[i][k]), to_host(w[i][k]),
                                   f"call {c} raster {i} ({src.width}x{src.height}, tile {tile}) output {k}")


def test_noalloc_rejects_oversized_and_host_rasters():
    ctx = engine.device_context(0)
    L = _lib.lib()
    spec = _set(13, 1)
    dsts = _outputs(spec)
    one, _keep = _c_items(spec, dsts)
    n = _lib.MAX_NOALLOC_BATCH + 1
    arr = (_lib.BatchItem * n)()
    for i in range(n):
        arr[i] = one[0]
    with pytest.raises(engine.StrataPanic, match="exceed"):
        _lib.check(L.strata_batch_run_noalloc(ctx, arr, n, None, 1))
    host_dst = [[like(spec[0][2]) for _ in range(spec[0][3])]]
    bad, _keep2 = _c_items(spec, host_dst)
    with pytest.raises(engine.StrataPanic, match="on the device"):
        _lib.check(L.strata_batch_run_noalloc(ctx, bad, 1, None, 1))
    # the scratch still serves a good call afterwards
    _lib.check(L.strata_batch_run_noalloc(ctx, one, 1, None, 1))
    want = _run_existing(ctx, spec)
    for k in range(spec[0][3]):
        assert_same_raster(to_host(dsts[0][k]), to_host(want[0][k]), f"after rejections, output {k}")


def test_noalloc_allocates_nothing_and_keeps_the_device():
    """After a first call (which looks the scratch up and loads the batch
    kernels), further calls leave the device's free memory exactly as it
    was: no cudaMalloc, no pool growth, no graph. The caller's current
    device is unchanged."""
    import torch

    ctx = engine.device_context(0)
    L = _lib.lib()
    spec = _set(14, 16)
    dsts = _outputs(spec)
    arr, _keep = _c_items(spec, dsts)
    _lib.check(L.strata_batch_run_noalloc(ctx, arr, len(spec), None, 1))
    torch.cuda.synchronize()
    dev = torch.cuda.current_device()
    free0 = torch.cuda.mem_get_info()[0]
    for i in range(20):
        _lib.check(L.strata_batch_run_noalloc(ctx, arr, len(spec), None, i % 2))
    _lib.check(L.strata_batch_run_noalloc(ctx, arr, len(spec), None, 1))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.current_device() == dev
    want = _run_existing(ctx, spec)
    for i, (_stages, _, src, nout, tile) in enumerate(spec):
        for k in range(nout):
            assert_same_raster(to_host(dsts[i][k]), to_host(want[i][k]), f"raster {i} output {k}")


def test_noalloc_refuses_a_capturing_stream():
    """A call on a stream that is being captured returns EINVAL (its
    descriptor copies come from host staging that the next call rewrites)
    and launches nothing."""
    import torch

    ctx = engine.device_context(0)
    L = _lib.lib()
    spec = _set(15, 2)
    dsts = _outputs(spec)
    arr, _keep = _c_items(spec, dsts)
    _lib.check(L.strata_batch_run_noalloc(ctx, arr, len(spec), None, 1))  # the scratch set up before capture
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    x = torch.zeros(16, device="cuda")
    rc = None
    with torch.cuda.graph(g, stream=s):
        x += 1
        rc = L.strata_batch_run_noalloc(ctx, arr, len(spec), s.cuda_stream, 0)
    assert rc == _lib.EINVAL
    assert "capturing" in _lib.last_error()
    del g
    # the scratch still serves an ordinary call
    _lib.check(L.strata_batch_run_noalloc(ctx, arr, len(spec), None, 1))
