"""The raw float32 file source and sink's host side (engine/raw.go): the
window reads and writes the chunked callbacks use when a raw file meets a
memory source or sink, the fill value as validity, and the checks. No
GPU: the device path is tests/test_gpu_raw.py."""
from __future__ import annotations

import numpy as np
import pytest

from strata_b200 import engine
from strata_b200.raster import Float32Raster, StrataPanic

FILL = np.float32(-9999)


def _file(tmp_path, cells, header=0):
    p = tmp_path / "r.f32"
    p.write_bytes(b"\x07" * header + np.ascontiguousarray(cells, "<f4").tobytes())
    return open(p, "r+b")


def _bits(m, off, n):
    b = np.unpackbits(np.asarray(m).view(np.uint8), bitorder="little")
    return b[off:off + n].astype(bool)


def test_read_window_fill_to_validity(tmp_path):
    rng = np.random.default_rng(1)
    h, w = 7, 11
    cells = rng.standard_normal((h, w)).astype(np.float32)
    cells[1, 2] = FILL
    cells[3, 4] = np.nan  # a NaN cell is valid when the fill is not NaN
    cells[5, 0] = -0.0
    with _file(tmp_path, cells, header=24) as f:
        src = engine.RawSource(f, w, h, engine.RawOptions(Fill=FILL, HasFill=True), offset=24)
        assert src.Masked() and src.Size() == (w, h)
        stride = 9
        dst = Float32Raster(np.zeros(stride * 4, np.float32), 6, 4, stride, np.zeros(2, np.uint64), 5)
        assert src.ReadWindow(dst, 1, 1) is None
        for y in range(4):
            got = dst.data[y * stride:y * stride + 6]
            assert (got.view(np.uint32) == cells[1 + y, 1:7].view(np.uint32)).all()
            ok = _bits(dst.valid, 5 + y * stride, 6)
            assert (ok == (cells[1 + y, 1:7] != FILL)).all()
        # zero as the fill matches -0 (by ==)
        z = engine.RawSource(f, w, h, engine.RawOptions(Fill=0.0, HasFill=True), offset=24)
        d2 = Float32Raster(np.zeros(w, np.float32), w, 1, w, np.zeros(1, np.uint64), 0)
        z.ReadWindow(d2, 0, 5)
        assert not _bits(d2.valid, 0, 1)[0]


def test_nan_fill_marks_every_nan(tmp_path):
    cells = np.array([[1, np.nan, 3], [np.float32(-np.nan), 5, 6]], np.float32)
    with _file(tmp_path, cells) as f:
        src = engine.RawSource(f, 3, 2, engine.RawOptions(Fill=np.nan, HasFill=True))
        d = Float32Raster(np.zeros(6, np.float32), 3, 2, 3, np.zeros(1, np.uint64), 0)
        src.ReadWindow(d, 0, 0)
        assert (_bits(d.valid, 0, 6) == np.array([1, 0, 1, 0, 1, 1], bool)).all()


def test_write_window_puts_fill_under_invalid_cells(tmp_path):
    h, w = 4, 5
    with _file(tmp_path, np.zeros((h, w), np.float32)) as f:
        sink = engine.RawSink(f, w, h, engine.RawOptions(Fill=FILL, HasFill=True))
        data = np.arange(12, dtype=np.float32)
        valid = np.zeros(1, np.uint64)
        bits = np.array([1, 0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 1], np.uint8)
        valid[0] = np.packbits(bits, bitorder="little").view(np.uint16)[0]
        src = Float32Raster(data, 3, 3, 4, valid, 0)
        assert sink.WriteWindow(src, 2, 1) is None
        f.seek(0)
        out = np.frombuffer(f.read(), "<f4").reshape(h, w)
        assert out[1, 2:5].tolist() == [0, FILL, 2]
        assert out[2, 2:5].tolist() == [4, 5, FILL]
        assert out[3, 2:5].tolist() == [8, 9, 10]
        assert src.data[1] == 1  # the caller's tile is left alone


def test_short_file_is_an_error(tmp_path):
    with _file(tmp_path, np.zeros((2, 4), np.float32)) as f:
        src = engine.RawSource(f, 4, 3, engine.RawOptions())
        d = Float32Raster(np.zeros(4, np.float32), 4, 1, 4)
        err = src.ReadWindow(d, 0, 2)
        assert isinstance(err, engine.SourceSinkError) and "row 2: unexpected EOF" in str(err)


def test_constructor_and_mask_checks(tmp_path):
    with pytest.raises(StrataPanic, match="dimensions must be positive, got 0×3"):
        engine.RawSource(0, 0, 3)
    with pytest.raises(StrataPanic, match="nil file"):
        engine.RawSink(None, 3, 3)
    with _file(tmp_path, np.zeros((2, 2), np.float32)) as f:
        src = engine.RawSource(f, 2, 2, engine.RawOptions(Fill=1, HasFill=True))
        with pytest.raises(StrataPanic, match="dst has no validity mask"):
            src.ReadWindow(Float32Raster(np.zeros(4, np.float32), 2, 2, 2), 0, 0)
        sink = engine.RawSink(f, 2, 2)
        with pytest.raises(StrataPanic, match="the sink has no fill value"):
            sink.WriteWindow(Float32Raster(np.zeros(4, np.float32), 2, 2, 2, np.zeros(1, np.uint64)), 0, 0)
