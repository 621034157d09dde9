"""The multi-GPU split on the device: row strips of one raster computed by
strata_process_strip equal the rows strata_process writes over the whole
raster, and strata_process_multi, run here over several contexts of the
one GPU (each its own stream and buffers, on threads of its own), equals
strata_process bit for bit, data and validity, with the strips' shared
mask words merged."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from helpers import assert_padding_untouched, assert_same_raster, host_raster, like, poison
from strata_b200 import _lib, engine, focal, shard, synth, terrain, transfer
from strata_b200.raster import Float32Raster, StrataPanic

pytestmark = pytest.mark.gpu


def dem(w, h, seed):
    return poison(synth.fbm_dem(w, h, seed, lo=0, hi=3000), seed, 0.003)


CASES = {
    "slope_reclass": lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10)).extend(
        transfer.reclass_stage([5, 10, 20], [1, 2, 3, 4])),
    "gradient": lambda: terrain.gradient_stage(terrain.GradientOptions(CellSize=10)),
    "curvature": lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=2)),
    "mean_r8": lambda: focal.box_stage(focal.BoxOptions(Radius=8), _lib.OP_MEAN),
    "tri_r3": lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=0, Radius=3)),
    "fit_aspect_r4": lambda: terrain.aspect_stage(terrain.AspectOptions(CellSize=10, FitRadius=4)),
    "rescale": lambda: transfer.rescale_stage(0.5, 1.0),
}


def nout_of(st):
    return 2 if st.stages[0].op == _lib.OP_GRADIENT else 1


def raster_pair(w, h, seed, masked):
    src = host_raster(dem(w, h, seed), synth.block_mask(w, h, seed, 0.05) if masked else None, w + 5, 13)
    return src


@pytest.mark.parametrize("name", sorted(CASES))
def test_strips_equal_whole_raster(name):
    rng = np.random.default_rng(len(name))
    for (w, h), masked in [((257, 131), True), ((130, 45), False), ((61, 300), True)]:
        src = raster_pair(w, h, w + h, masked)
        st = CASES[name]
        n = nout_of(st())
        want = [like(src, w + 3, 7) for _ in range(n)]
        assert engine.process(st(), want, [src]) is None
        got = [like(src, w + 3, 7) for _ in range(n)]
        before = [Float32Raster(np.array(g.data), g.width, g.height, g.stride,
                                None if g.valid is None else np.array(g.valid), g.valid_offset) for g in got]
        r = shard.stage_radius(st())
        cuts = sorted(set([0, h] + list(rng.integers(1, h, 3))))
        for y0, y1 in zip(cuts[:-1], cuts[1:]):
            s0, s1 = shard.halo_rows(h, r, y0, y1)
            # extra source rows beyond the halo are allowed too
            s0, s1 = max(0, s0 - int(rng.integers(0, 3))), min(h, s1 + int(rng.integers(0, 3)))
            engine.process_strip(st(), [g.Window(0, y0, w, y1 - y0) for g in got], src.Window(0, s0, w, s1 - s0), h,
                                 s0, y0)
        for i in range(n):
            assert_same_raster(got[i], want[i], f"{name} {w}x{h} cuts={cuts} out{i}")
            assert_padding_untouched(before[i], got[i], f"{name} out{i}")


def _contexts(k):
    out = []
    for _ in range(k):
        p = ctypes.c_void_p()
        _lib.check(_lib.lib().strata_ctx_create(0, ctypes.byref(p)))
        out.append(p)
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_multi_over_contexts_equals_process(name):
    ctxs = _contexts(3)
    try:
        for (w, h), masked in [((300, 97), True), ((1030, 64), True), ((77, 5), False)]:
            src = raster_pair(w, h, w * h, masked)
            st = CASES[name]
            n = nout_of(st())
            want = [like(src, w + 2, 33) for _ in range(n)]
            assert engine.process(st(), want, [src]) is None
            got = [like(src, w + 2, 33) for _ in range(n)]
            s = st()
            arr = (ctypes.c_void_p * 3)(*ctxs)
            srcs = (_lib.Raster * 1)(engine.c_raster(src))
            dsts = (_lib.Raster * n)(*[engine.c_raster(g) for g in got])
            o = _lib.ExecOpts()
            cst = _lib.Stats()
            _lib.check(_lib.lib().strata_process_multi(arr, 3, s.c_array(), len(s.stages), srcs, 1, dsts, n,
                                                       ctypes.byref(o), ctypes.byref(cst)))
            assert cst.cells == w * h
            for i in range(n):
                assert_same_raster(got[i], want[i], f"multi {name} {w}x{h} out{i}")
    finally:
        for c in ctxs:
            _lib.lib().strata_ctx_destroy(c)


def test_devices_option_and_sharded_single_rank():
    w, h = 400, 150
    src = raster_pair(w, h, 3, True)
    st = lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10))
    want = like(src)
    engine.process(st(), [want], [src])
    got = like(src)
    assert engine.process(st(), [got], [src], engine.Options(Devices=[0, 0])) is None
    assert_same_raster(got, want, "Devices=[0, 0]")
    got2 = like(src)
    shard.process_sharded(st(), [got2], src, 0, 1)
    assert_same_raster(got2, want, "process_sharded world 1")


def test_strip_checks():
    w, h = 64, 40
    src = raster_pair(w, h, 1, False)
    dst = like(src)
    st = lambda: focal.box_stage(focal.BoxOptions(Radius=4), _lib.OP_MEAN)
    with pytest.raises(StrataPanic, match="do not cover"):
        engine.process_strip(st(), [dst.Window(0, 10, w, 10)], src.Window(0, 8, w, 14), h, 8, 10)
    with pytest.raises(StrataPanic, match="must lie in the raster"):
        engine.process_strip(st(), [dst.Window(0, 30, w, 10)], src.Window(0, 26, w, 14), 35, 26, 30)
    d2 = like(src)
    with pytest.raises(StrataPanic, match="no cancellable context"):
        engine.process_multi(st(), [d2], [src], engine.Options(Devices=[0, 0]), engine.Background())
