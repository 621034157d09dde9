"""Chunked processing of raw float32 files on the device (engine/raw.go with
exec.ProcessChunked): tiles read with pread, the fill value turned into
validity on the device and put back under invalid output cells on the
device, tiles written with pwrite; against the oracle on the same raster
held in memory, the output file compared cell for cell (rastertest.
SameFloat), and against the host-side callback path."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import host_raster, like, poison, run_oracle, same_bits
from strata_b200 import algebra, engine, focal, synth, terrain, transfer
from strata_b200.raster import StrataPanic

pytestmark = pytest.mark.gpu

FILL = np.float32(-9999.0)


def dem(w, h, seed, holes=0.02, fill=FILL):
    c = poison(synth.fbm_dem(w, h, seed, lo=0, hi=3000), seed, 0.002)
    m = synth.block_mask(w, h, seed, holes)
    c = c.copy()
    c[~m] = fill
    return c


def write_file(path, cells, header=0):
    path.write_bytes(b"\xab" * header + np.ascontiguousarray(cells, "<f4").tobytes())
    return path


def read_file(path, w, h, header=0):
    return np.frombuffer(path.read_bytes()[header:header + 4 * w * h], "<f4").reshape(h, w)


def expected(stages, cells, fill, out_fill, nout=1):
    """The oracle over the raster in memory, its mask from the fill value
    (RawSource), the fill put under invalid output cells (RawSink)."""
    h, w = cells.shape
    valid = None
    if fill is not None:
        valid = (~np.isnan(cells)) if np.isnan(fill) else (cells != fill)
    src = host_raster(cells, valid)
    outs = [like(src, masked=fill is not None or out_fill is not None) for _ in range(nout)]
    run_oracle(stages, src, outs)
    res = []
    for o in outs:
        a = o.numpy().copy()
        if out_fill is not None:
            a[~o.valid_numpy()] = out_fill
        res.append(a)
    return res


def check_same(got, want, what):
    ok = same_bits(got, want)
    if not ok.all():
        ys, xs = np.nonzero(~ok)
        raise AssertionError(f"{what}: {int((~ok).sum())} cells differ, first at ({xs[0]}, {ys[0]}): "
                             f"got {got[ys[0], xs[0]]!r} want {want[ys[0], xs[0]]!r}")


PIPES = {
    "slope_lookup_reclass": (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10)).extend(
        transfer.lookup_stage([0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5])).extend(
        transfer.reclass_stage([1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5])), 1),
    "gradient": (lambda: terrain.gradient_stage(terrain.GradientOptions(CellSize=10)), 2),
    "mean_r5": (lambda: focal.box_stage(focal.BoxOptions(Radius=5), engine._lib.OP_MEAN), 1),
    "hillshade_clamp": (lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10)).extend(
        algebra.clamp_stage(50, 200)), 1),
    "rescale_alone": (lambda: transfer.rescale_stage(0.5, -3), 1),
}


@pytest.mark.parametrize("name", sorted(PIPES))
@pytest.mark.parametrize("tiles", [(0, 0), (256, 96), (1000, 37)])
def test_raw_files_as_the_oracle(tmp_path, name, tiles):
    make, nout = PIPES[name]
    w, h = 1031, 300
    cells = dem(w, h, len(name) + tiles[0])
    hdr = 40
    src_path = write_file(tmp_path / "dem.f32", cells, hdr)
    outs = [tmp_path / f"out{i}.f32" for i in range(nout)]
    out_fill = np.float32(-1.0)
    with open(src_path, "rb") as f:
        files = [open(p, "w+b") for p in outs]
        try:
            src = engine.RawSource(f, w, h, engine.RawOptions(Fill=FILL, HasFill=True), offset=hdr)
            sinks = [engine.RawSink(g, w, h, engine.RawOptions(Fill=out_fill, HasFill=True), offset=8) for g in files]
            st = engine.Stats()
            assert engine.process_chunked(make(), sinks, [src],
                                          engine.Options(TileWidth=tiles[0], TileHeight=tiles[1], Stats=st)) is None
        finally:
            for g in files:
                g.close()
    want = expected(make(), cells, FILL, out_fill, nout)
    for i, p in enumerate(outs):
        check_same(read_file(p, w, h, 8), want[i], f"{name} tiles={tiles} out{i}")
    assert st.SourceRead >= w * h * 4 and st.SinkWritten == w * h * 4 * nout


def test_nan_and_zero_fills(tmp_path):
    w, h = 300, 70
    for fill in (np.float32(np.nan), np.float32(0.0)):
        cells = dem(w, h, 3, fill=fill)
        if fill == 0:
            cells[5, 5:9] = -0.0  # -0 matches a zero fill
        p = write_file(tmp_path / "a.f32", cells)
        q = tmp_path / "b.f32"
        with open(p, "rb") as f, open(q, "w+b") as g:
            assert engine.process_chunked(terrain.slope_stage(terrain.SlopeOptions(CellSize=10)),
                                          [engine.RawSink(g, w, h, engine.RawOptions(Fill=fill, HasFill=True))],
                                          [engine.RawSource(f, w, h, engine.RawOptions(Fill=fill, HasFill=True))],
                                          engine.Options(TileWidth=128, TileHeight=32)) is None
        want = expected(terrain.slope_stage(terrain.SlopeOptions(CellSize=10)), cells, fill, fill)[0]
        check_same(read_file(q, w, h), want, f"fill={fill}")


def test_unmasked_files(tmp_path):
    """No fill on either side: every cell valid, the edge ring NaN."""
    w, h = 517, 41
    cells = dem(w, h, 4, holes=0.0)
    p = write_file(tmp_path / "a.f32", cells)
    q = tmp_path / "b.f32"
    with open(p, "rb") as f, open(q, "w+b") as g:
        assert engine.process_chunked(terrain.aspect_stage(terrain.AspectOptions(CellSize=5)),
                                      [engine.RawSink(g, w, h)], [engine.RawSource(f, w, h)],
                                      engine.Options(TileHeight=16)) is None
    want = expected(terrain.aspect_stage(terrain.AspectOptions(CellSize=5)), cells, None, None)[0]
    check_same(read_file(q, w, h), want, "unmasked")


def test_raw_source_into_memory_sink_equals_device_path(tmp_path):
    """A raw source with a memory sink goes through the host callbacks; its
    cells and validity equal the device path's."""
    w, h = 640, 200
    cells = dem(w, h, 5)
    p = write_file(tmp_path / "a.f32", cells)
    st = lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10))
    mem = like(host_raster(cells, np.ones((h, w), bool)))
    with open(p, "rb") as f:
        src = engine.RawSource(f, w, h, engine.RawOptions(Fill=FILL, HasFill=True))
        assert engine.process_chunked(st(), [engine.MemorySink(mem)], [src],
                                      engine.Options(TileWidth=300, TileHeight=64)) is None
    valid = cells != FILL
    want = like(mem)
    run_oracle(st(), host_raster(cells, valid), [want])
    check_same(mem.numpy(), want.numpy(), "memory sink")
    assert (mem.valid_numpy() == want.valid_numpy()).all()


def test_errors(tmp_path):
    w, h = 64, 32
    p = write_file(tmp_path / "short.f32", np.zeros((h - 3, w), np.float32))
    q = tmp_path / "o.f32"
    with open(p, "rb") as f, open(q, "w+b") as g:
        err = engine.process_chunked(terrain.slope_stage(terrain.SlopeOptions(CellSize=1)), [engine.RawSink(g, w, h)],
                                     [engine.RawSource(f, w, h)], engine.Options(TileHeight=8))
        assert isinstance(err, engine.SourceSinkError) and "unexpected EOF" in str(err), err
        with pytest.raises(StrataPanic, match="its validity would be lost"):
            engine.process_chunked(terrain.slope_stage(terrain.SlopeOptions(CellSize=1)), [engine.RawSink(g, w, h)],
                                   [engine.RawSource(f, w, h, engine.RawOptions(Fill=0, HasFill=True))])
