"""Shared test helpers: rasters from numpy, the oracle on the same inputs,
and the reference's comparison rule (rastertest.SameFloat,
internal/rastertest/rastertest.go:181-184: same bits, or both NaN)."""
from __future__ import annotations

import numpy as np

from oracle import oracle as orc
from strata_b200 import _lib
from strata_b200.raster import Float32Raster, mask_from_bool

NAN = np.float32("nan")


def host_raster(cells: np.ndarray, valid=None, stride=None, offset=0, pad_value=np.float32(-7.5)) -> Float32Raster:
    """A host raster holding cells (h, w), with an optional bool mask, a
    stride >= w (padding cells filled with pad_value) and a bit offset."""
    h, w = cells.shape
    stride = w if stride is None else stride
    data = np.full((h - 1) * stride + w, pad_value, np.float32)
    for y in range(h):
        data[y * stride:y * stride + w] = cells[y]
    m = None
    if valid is not None:
        m = mask_from_bool(valid, stride, offset)
        # set the padding bits so a bug that reads them shows
        m |= ~mask_from_bool(np.ones_like(valid), stride, offset, words=len(m)) & np.uint64(0x5555555555555555)
    return Float32Raster(data, w, h, stride, m, offset)


def like(r: Float32Raster, stride=None, offset=0, fill=np.float32(1234.5), masked=None) -> Float32Raster:
    """An output raster for r, pre-filled with garbage so unwritten cells show."""
    h, w = r.height, r.width
    stride = w if stride is None else stride
    data = np.full((h - 1) * stride + w, fill, np.float32)
    m = None
    if (r.valid is not None) if masked is None else masked:
        n = offset + (h - 1) * stride + w
        m = np.full((n + 63) // 64, np.uint64(0xA5A5A5A5A5A5A5A5), dtype=np.uint64)
    return Float32Raster(data, w, h, stride, m, offset)


def to_device(r: Float32Raster) -> Float32Raster:
    import torch

    d = torch.from_numpy(np.asarray(r.data).copy()).cuda()
    v = None
    if r.valid is not None:
        v = torch.from_numpy(np.asarray(r.valid).view(np.int64).copy()).cuda()
    return Float32Raster(d, r.width, r.height, r.stride, v, r.valid_offset)


def to_host(r: Float32Raster) -> Float32Raster:
    if not r.on_device():
        return r
    d = r.data.cpu().numpy()
    v = r.valid.cpu().numpy().view(np.uint64) if r.valid is not None else None
    return Float32Raster(d, r.width, r.height, r.stride, v, r.valid_offset)


def _orc_dict(r: Float32Raster):
    return dict(data=r.data, width=r.width, height=r.height, stride=r.stride,
                valid=r.valid, valid_offset=r.valid_offset)


def oracle_stage(st: _lib.Stage):
    """The oracle stage equal to a product stage (Convolve's rotation, which
    focal/correlate.go:80-86 applies on the host, applied here)."""
    # Tables keep their slots: an empty one (a Reclass with no breaks) is
    # an empty array ahead of the later ones.
    tables = []
    for i in range(4):
        n = st.table_len[i]
        if st.table[i] and n > 0:
            tables.append(np.ctypeslib.as_array((np.ctypeslib.ctypes.c_float * n).from_address(st.table[i])).copy())
        else:
            tables.append(np.zeros(0, np.float32))
    while tables and tables[-1].size == 0:
        tables.pop()
    if st.op == _lib.OP_CORRELATE and st.flags & _lib.STAGE_ROTATE180:
        tables[0] = tables[0][::-1].copy()
    return orc.stage(st.op, st.radius, st.kind, list(st.k), tables, flags=st.flags & _lib.STAGE_FIT, input=st.input)


def run_oracle(stages, src, dsts, nthreads=1):
    """Runs the oracle for a product StageList into host rasters dsts; src
    is one raster, or a list of them for a pointwise chain."""
    ost = [oracle_stage(s) for s in stages.stages]
    if isinstance(src, (list, tuple)):
        orc.process_n(ost, [_orc_dict(x) for x in src], [_orc_dict(d) for d in dsts], nthreads)
        return
    orc.process(ost, _orc_dict(src), [_orc_dict(d) for d in dsts], nthreads)


def same_bits(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-cell SameFloat: identical bits, or both NaN."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))


def assert_same_raster(got: Float32Raster, want: Float32Raster, what=""):
    got, want = to_host(got), to_host(want)
    g, w = got.numpy(), want.numpy()
    ok = same_bits(g, w)
    if not ok.all():
        ys, xs = np.nonzero(~ok)
        y, x = ys[0], xs[0]
        raise AssertionError(
            f"{what}: {int((~ok).sum())} cells differ; first at ({x}, {y}): got {g[y, x]!r} "
            f"({g[y, x:x+1].view(np.uint32)[0]:#010x}), want {w[y, x]!r} ({w[y, x:x+1].view(np.uint32)[0]:#010x})")
    gv, wv = got.valid_numpy(), want.valid_numpy()
    assert (gv is None) == (wv is None), f"{what}: mask presence differs"
    if gv is not None:
        bad = gv != wv
        if bad.any():
            ys, xs = np.nonzero(bad)
            raise AssertionError(f"{what}: {int(bad.sum())} validity bits differ; first at ({xs[0]}, {ys[0]}): "
                                 f"got {gv[ys[0], xs[0]]}, want {wv[ys[0], xs[0]]}")


def assert_padding_untouched(before: Float32Raster, after: Float32Raster, what=""):
    """Cells outside the raster's own (gap cells of a stride) and mask bits
    outside its span are left alone."""
    a = np.asarray(to_host(after).data)
    b = np.asarray(before.data)
    for y in range(before.height - 1):
        s = y * before.stride + before.width
        e = (y + 1) * before.stride
        assert same_bits(a[s:e], b[s:e]).all(), f"{what}: padding cells of row {y} changed"
    if before.valid is not None:
        bv = np.unpackbits(np.asarray(before.valid).view(np.uint8), bitorder="little")
        av = np.unpackbits(np.asarray(to_host(after).valid).view(np.uint8), bitorder="little")
        own = np.zeros(bv.size, bool)
        for y in range(before.height):
            s = before.valid_offset + y * before.stride
            own[s:s + before.width] = True
        assert (bv[~own] == av[~own]).all(), f"{what}: mask bits outside the raster changed"


def poison(cells: np.ndarray, seed: int, frac=0.01) -> np.ndarray:
    """Scatters NaN, +-Inf, -0, +0 and subnormals over a copy of cells."""
    out = cells.copy()
    rng = np.random.default_rng(seed)
    n = out.size
    k = max(1, int(n * frac))
    idx = rng.choice(n, size=min(k, n), replace=False)
    specials = np.array([np.nan, np.inf, -np.inf, -0.0, 0.0, 1e-40, -1e-42, 3.4e38], np.float32)
    out.reshape(-1)[idx] = specials[rng.integers(0, specials.size, idx.size)]
    return out
