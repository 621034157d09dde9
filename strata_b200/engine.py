"""engine: options, statistics, sources and sinks, and the drivers that run
a stage list on the device (strata's engine package, engine/engine.go,
engine/stats.go, engine/source.go, and internal/exec's ProcessN /
ProcessChunked, internal/exec/process.go:28 and chunked.go:33).

The drivers hand the whole call to libstrata_cuda (strata_process /
strata_process_chunked); nothing here computes cells.
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .raster import Float32Raster, StrataPanic, _is_torch

BYTES_PER_CELL = 4


@dataclass
class Options:
    """engine.Options (engine/engine.go:7-28). TileWidth / TileHeight pick
    the chunked tiles (0 = the whole raster); Workers is accepted for
    parity. Stats, when set, is added to by the call. Stream is an optional
    torch.cuda.Stream for device-resident operands; Async skips the final
    synchronisation when every operand is on the device. Device picks the
    GPU; Devices, with more than one entry, splits a plain call's raster
    into row strips over those GPUs (strata_process_multi)."""
    TileWidth: int = 0
    TileHeight: int = 0
    Workers: int = 0
    Stats: Optional["Stats"] = None
    Stream: object = None
    Async: bool = False
    Device: int = 0
    Devices: Optional[List[int]] = None


@dataclass
class Stats:
    """engine.Stats (engine/stats.go:77-168), for the device's tiling."""
    Cells: int = 0
    Ideal: int = 0
    Tiles: int = 0
    Bands: int = 0
    SourceRead: int = 0
    SinkWritten: int = 0
    KernelRead: int = 0
    KernelWritten: int = 0

    def Total(self) -> int:
        return self.SourceRead + self.KernelRead + self.KernelWritten + self.SinkWritten

    def Amplification(self) -> float:
        return 0.0 if self.Ideal == 0 else self.Total() / self.Ideal

    def BytesPerCell(self) -> float:
        return 0.0 if self.Cells == 0 else self.Total() / self.Cells

    def Halo(self, inputs: int) -> int:
        return 0 if inputs <= 0 else self.KernelRead - self.Cells * BYTES_PER_CELL * inputs

    def Add(self, o: "Stats") -> None:
        for f in ("Cells", "Ideal", "Tiles", "Bands", "SourceRead", "SinkWritten", "KernelRead", "KernelWritten"):
            setattr(self, f, getattr(self, f) + getattr(o, f))


class Canceled(Exception):
    """The Context was cancelled before every cell was written (ctx.Err())."""


class SourceSinkError(IOError):
    """A source or sink failed; the call stopped after a plan-order prefix."""


class Context:
    """A cancellation context (Go's context.Context, for the Tiled and
    Chunked entry points): cancel() stops a running call between strips or
    tiles."""

    def __init__(self):
        self._flag = ctypes.c_int32(0)

    def cancel(self) -> None:
        self._flag.value = 1

    def Err(self):
        return Canceled("context canceled") if self._flag.value else None


def Background() -> Context:
    return Context()


# ---------------------------------------------------------------------------
# Device contexts, one per device, created on first use.

_ctx_lock = threading.Lock()
_ctxs = {}


def device_context(device: int = 0):
    with _ctx_lock:
        c = _ctxs.get(device)
        if c is None:
            p = ctypes.c_void_p()
            _lib.check(_lib.lib().strata_ctx_create(device, ctypes.byref(p)))
            c = p
            _ctxs[device] = c
        return c


def _ptr(a) -> int:
    if _is_torch(a):
        return a.data_ptr()
    return a.ctypes.data


def c_raster(r: Float32Raster) -> _lib.Raster:
    """The C view of a raster (no copy)."""
    r.Validate()
    out = _lib.Raster()
    out.data = _ptr(r.data)
    out.width, out.height, out.stride = r.width, r.height, r.stride
    out.valid = _ptr(r.valid) if r.valid is not None else None
    out.valid_offset = r.valid_offset
    dev = r.on_device()
    if r.valid is not None and _is_torch(r.valid) != dev:
        raise StrataPanic("engine: a raster's Data and Valid must be in the same memory (host or device)")
    if not dev and not (isinstance(r.data, np.ndarray) and r.data.dtype == np.float32):
        raise StrataPanic("engine: host Data must be a float32 numpy array")
    out.on_device = 1 if dev else 0
    return out


def c_opts(opts: Optional[Options], ctx: Optional[Context] = None) -> _lib.ExecOpts:
    o = _lib.ExecOpts()
    if opts is not None:
        o.tile_width, o.tile_height, o.workers = opts.TileWidth, opts.TileHeight, opts.Workers
        o.flags = _lib.EXEC_ASYNC if opts.Async else 0
        if opts.Stream is not None:
            o.stream = getattr(opts.Stream, "cuda_stream", opts.Stream)
    if ctx is not None:
        o.cancel = ctypes.pointer(ctx._flag)
    return o


class StageList:
    """Stages plus the host arrays their tables point into."""

    def __init__(self):
        self.stages: List[_lib.Stage] = []
        self.keep: list = []
        self._c = None

    def add(self, st: _lib.Stage, *arrays) -> "StageList":
        self.stages.append(st)
        self.keep.extend(arrays)
        self._c = None
        return self

    def extend(self, other: "StageList") -> "StageList":
        self.stages.extend(other.stages)
        self.keep.extend(other.keep)
        self._c = None
        return self

    def c_array(self):
        return (_lib.Stage * len(self.stages))(*self.stages)

    def c_address(self) -> int:
        """The address of the stages as a C array, built once and kept with
        the list until stages are added (for calls that pass many lists)."""
        if self._c is None:
            arr = self.c_array()
            self._c = (arr, ctypes.addressof(arr))
        return self._c[1]


def _stats_out(opts: Optional[Options], cst: _lib.Stats) -> None:
    if opts is not None and opts.Stats is not None:
        opts.Stats.Add(Stats(cst.cells, cst.ideal, cst.tiles, cst.bands, cst.source_read,
                             cst.sink_written, cst.kernel_read, cst.kernel_written))


def process(stages: StageList, dst: Sequence[Float32Raster], src: Sequence[Float32Raster],
            opts: Optional[Options] = None, ctx: Optional[Context] = None):
    """exec.ProcessN on the device. Returns None, or Canceled if ctx was
    cancelled first; raises StrataPanic on programming errors."""
    if opts is not None and opts.Devices and len(opts.Devices) > 1:
        return process_multi(stages, dst, src, opts, ctx)
    dev = opts.Device if opts is not None else 0
    c = device_context(dev)
    srcs = (_lib.Raster * len(src))(*[c_raster(s) for s in src])
    dsts = (_lib.Raster * len(dst))(*[c_raster(d) for d in dst])
    o = c_opts(opts, ctx)
    cst = _lib.Stats()
    rc = _lib.lib().strata_process(c, stages.c_array(), len(stages.stages), srcs, len(src), dsts, len(dst),
                                   ctypes.byref(o), ctypes.byref(cst))
    _stats_out(opts, cst)
    if rc == _lib.ECANCELED:
        return Canceled("context canceled")
    _lib.check(rc)
    return None


def process_multi(stages: StageList, dst: Sequence[Float32Raster], src: Sequence[Float32Raster],
                  opts: Options, ctx: Optional[Context] = None):
    """A plain call split into row strips over opts.Devices, each strip with
    its halo rows computed on its own GPU (strata_process_multi); the same
    bits as one device. Host rasters."""
    if ctx is not None:
        raise StrataPanic("engine: a multi-device call takes no cancellable context")
    ctxs = (ctypes.c_void_p * len(opts.Devices))(*[device_context(d) for d in opts.Devices])
    srcs = (_lib.Raster * len(src))(*[c_raster(s) for s in src])
    dsts = (_lib.Raster * len(dst))(*[c_raster(d) for d in dst])
    o = c_opts(Options(TileWidth=opts.TileWidth, TileHeight=opts.TileHeight, Workers=opts.Workers))
    cst = _lib.Stats()
    rc = _lib.lib().strata_process_multi(ctxs, len(opts.Devices), stages.c_array(), len(stages.stages), srcs,
                                         len(src), dsts, len(dst), ctypes.byref(o), ctypes.byref(cst))
    _stats_out(opts, cst)
    _lib.check(rc)
    return None


def process_strip(stages: StageList, dst: Sequence[Float32Raster], src: Float32Raster, height: int, src_row: int,
                  dst_row: int, opts: Optional[Options] = None):
    """Rows [dst_row, dst_row + dst[0].height) of a height-row raster's
    outputs from its input rows [src_row, src_row + src.height), as
    strata_process writes them over the whole raster (strata_process_strip)."""
    dev = opts.Device if opts is not None else 0
    c = device_context(dev)
    s = c_raster(src)
    dsts = (_lib.Raster * len(dst))(*[c_raster(d) for d in dst])
    strip = _lib.Strip(height, src_row, dst_row)
    o = c_opts(opts)
    cst = _lib.Stats()
    rc = _lib.lib().strata_process_strip(c, stages.c_array(), len(stages.stages), ctypes.byref(s), dsts, len(dst),
                                         ctypes.byref(strip), ctypes.byref(o), ctypes.byref(cst))
    _stats_out(opts, cst)
    _lib.check(rc)
    return None


def process_features(features: Sequence[StageList], dst: Sequence[Float32Raster], src: Float32Raster,
                     opts: Optional[Options] = None, ctx: Optional[Context] = None):
    """Several pipelines over one input in one call (terrain.Features,
    terrain.Surface): features[i] writes the next outputs of dst (two for a
    gradient). A host input crosses to the device once. Returns None;
    raises StrataPanic on programming errors."""
    dev = opts.Device if opts is not None else 0
    c = device_context(dev)
    all_stages = StageList()
    counts = []
    for f in features:
        all_stages.extend(f)
        counts.append(len(f.stages))
    cnt = (ctypes.c_int32 * len(counts))(*counts)
    srcs = (_lib.Raster * 1)(c_raster(src))
    dsts = (_lib.Raster * len(dst))(*[c_raster(d) for d in dst])
    o = c_opts(opts, ctx)
    cst = _lib.Stats()
    rc = _lib.lib().strata_process_features(c, all_stages.c_array(), cnt, len(counts), srcs, dsts, len(dst),
                                            ctypes.byref(o), ctypes.byref(cst))
    _stats_out(opts, cst)
    if rc == _lib.ECANCELED:
        return Canceled("context canceled")
    _lib.check(rc)
    return None


# ---------------------------------------------------------------------------
# Sources and sinks (engine/source.go).

class RasterSource:
    """engine.RasterSource: Size(), Masked(), ReadWindow(dst, x, y)."""

    def Size(self):
        raise NotImplementedError

    def Masked(self) -> bool:
        raise NotImplementedError

    def ReadWindow(self, dst: Float32Raster, x: int, y: int):
        raise NotImplementedError


class RasterSink:
    """engine.RasterSink: Size(), Masked(), WriteWindow(src, x, y)."""

    def Size(self):
        raise NotImplementedError

    def Masked(self) -> bool:
        raise NotImplementedError

    def WriteWindow(self, src: Float32Raster, x: int, y: int):
        raise NotImplementedError


def _copy_cells(dst: Float32Raster, src: Float32Raster, valid: bool) -> None:
    for y in range(dst.height):
        dst.data[y * dst.stride:y * dst.stride + dst.width] = src.data[y * src.stride:y * src.stride + dst.width]
    if valid:
        _copy_validity(dst, src)


def _bits(m, off: int, n: int) -> np.ndarray:
    w0 = off >> 6
    w1 = (off + n + 63) >> 6
    b = np.unpackbits(np.asarray(m[w0:w1]).view(np.uint8), bitorder="little")
    s = off - w0 * 64
    return b[s:s + n]


def _put_bits(m, off: int, bits: np.ndarray) -> None:
    n = len(bits)
    if n == 0:
        return
    w0 = off >> 6
    w1 = (off + n + 63) >> 6
    cur = np.unpackbits(np.asarray(m[w0:w1]).view(np.uint8), bitorder="little")
    s = off - w0 * 64
    cur[s:s + n] = bits
    m[w0:w1] = np.packbits(cur, bitorder="little").view(np.uint64)


def _copy_validity(dst: Float32Raster, src: Float32Raster) -> None:
    for y in range(dst.height):
        if src.valid is None:
            bits = np.ones(dst.width, np.uint8)
        else:
            bits = _bits(src.valid, src.valid_offset + y * src.stride, dst.width)
        _put_bits(dst.valid, dst.valid_offset + y * dst.stride, bits)


class MemorySource(RasterSource):
    """engine.MemorySource (engine/source.go:72-104): windows of a host raster."""

    def __init__(self, r: Float32Raster):
        r.Validate()
        self.r = r

    def Raster(self):
        return self.r

    def Size(self):
        return self.r.width, self.r.height

    def Masked(self) -> bool:
        return self.r.valid is not None

    def ReadWindow(self, dst: Float32Raster, x: int, y: int):
        if self.r.valid is not None and dst.valid is None:
            raise StrataPanic("engine: MemorySource.ReadWindow: the source has a validity mask and dst has none")
        _copy_cells(dst, self.r.Window(x, y, dst.width, dst.height), dst.valid is not None)
        return None


class MemorySink(RasterSink):
    """engine.MemorySink (engine/source.go:106-144): writes into a host raster."""

    def __init__(self, r: Float32Raster):
        r.Validate()
        self.r = r

    def Raster(self):
        return self.r

    def Size(self):
        return self.r.width, self.r.height

    def Masked(self) -> bool:
        return self.r.valid is not None

    def WriteWindow(self, src: Float32Raster, x: int, y: int):
        if src.valid is not None and self.r.valid is None:
            raise StrataPanic("engine: MemorySink.WriteWindow: src has a validity mask and the sink has none")
        dst = self.r.Window(x, y, src.width, src.height)
        _copy_cells(dst, src, False)
        if dst.valid is not None:
            _copy_validity(dst, src)
        return None


def _buffer_view(b: _lib.Raster) -> Float32Raster:
    n = (b.height - 1) * b.stride + b.width
    data = np.ctypeslib.as_array(ctypes.cast(b.data, ctypes.POINTER(ctypes.c_float)), shape=(n,))
    valid = None
    if b.valid:
        words = (b.valid_offset + n + 63) // 64
        valid = np.ctypeslib.as_array(ctypes.cast(b.valid, ctypes.POINTER(ctypes.c_uint64)), shape=(words,))
    return Float32Raster(data, b.width, b.height, b.stride, valid, b.valid_offset)


def process_chunked(stages: StageList, dst: Sequence[RasterSink], src: Sequence[RasterSource],
                    opts: Optional[Options] = None, ctx: Optional[Context] = None):
    """exec.ProcessChunked on the device. Returns None, Canceled, or the
    first source / sink error (a SourceSinkError wrapping it). With raw
    files on every side it runs process_raw."""
    if src and dst and all(isinstance(s, RawSource) for s in src) and all(isinstance(d, RawSink) for d in dst):
        return process_raw(stages, dst, src, opts, ctx)
    dev = opts.Device if opts is not None else 0
    c = device_context(dev)
    errors: list = []

    def reader(j):
        def f(user, buf, x, y):
            try:
                err = src[j].ReadWindow(_buffer_view(buf.contents), x, y)
            except StrataPanic:
                raise
            except Exception as e:  # a failing source
                err = e
            if err is not None:
                errors.append(SourceSinkError(f"engine: reading src[{j}] at ({x}, {y}): {err}"))
                return 1
            return 0
        return _lib.READ_FN(f)

    def writer(j):
        def f(user, buf, x, y):
            try:
                err = dst[j].WriteWindow(_buffer_view(buf.contents), x, y)
            except StrataPanic:
                raise
            except Exception as e:
                err = e
            if err is not None:
                errors.append(SourceSinkError(f"engine: writing dst[{j}] at ({x}, {y}): {err}"))
                return 1
            return 0
        return _lib.WRITE_FN(f)

    cbs = []
    srcs = (_lib.Source * len(src))()
    for j, s in enumerate(src):
        w, h = s.Size()
        cb = reader(j)
        cbs.append(cb)
        srcs[j].width, srcs[j].height, srcs[j].masked = w, h, 1 if s.Masked() else 0
        srcs[j].read = cb
    dsts = (_lib.Sink * len(dst))()
    for j, d in enumerate(dst):
        w, h = d.Size()
        cb = writer(j)
        cbs.append(cb)
        dsts[j].width, dsts[j].height, dsts[j].masked = w, h, 1 if d.Masked() else 0
        dsts[j].write = cb
    o = c_opts(opts, ctx)
    cst = _lib.Stats()
    rc = _lib.lib().strata_process_chunked(c, stages.c_array(), len(stages.stages), srcs, len(src), dsts,
                                           len(dst), ctypes.byref(o), ctypes.byref(cst))
    _stats_out(opts, cst)
    if rc == _lib.ECANCELED:
        return Canceled("context canceled")
    if rc == _lib.EIO:
        return errors[0] if errors else SourceSinkError(_lib.last_error())
    _lib.check(rc)
    return None


# ---------------------------------------------------------------------------
# Raw float32 files (engine/raw.go): little-endian cells, row-major, no
# header, at a byte offset of an open file. A chunked call whose sources
# and sinks are all raw files runs strata_process_raw: the tiles are read
# with pread into page-locked memory, their validity is taken from the fill
# value on the device, the fill goes under the invalid output cells on the
# device, and the tiles are written with pwrite. Mixed with other sources
# or sinks, the raw ones serve windows through ReadWindow / WriteWindow
# on the host (the same bits).

@dataclass
class RawOptions:
    """engine.RawOptions: Fill is the file's NoData value when HasFill."""
    Fill: float = 0.0
    HasFill: bool = False


def _raw_size_check(fn: str, f, width: int, height: int) -> None:
    if f is None:
        raise StrataPanic(f"engine: {fn}: nil file")
    if width <= 0 or height <= 0:
        raise StrataPanic(f"engine: {fn}: dimensions must be positive, got {width}×{height}")
    if width > ((1 << 63) - 1) // 4 // height:
        raise StrataPanic(f"engine: {fn}: {width}×{height} cells do not fit in a file")


def _fd(f) -> int:
    return f if isinstance(f, int) else f.fileno()


def _rows(r: Float32Raster, width: int):
    """(first row, rows) groups of r one call moves: all rows at once when
    they are consecutive in the file and in r, else one a call."""
    per = r.height if (r.width == width and r.stride == r.width) else 1
    for row in range(0, r.height, per):
        yield row, min(per, r.height - row)


def _rows_name(y: int, k: int) -> str:
    return f"row {y}" if k == 1 else f"rows {y} to {y + k - 1}"


class RawSource(RasterSource):
    """engine.RawSource: a width×height raw float32 raster read from f (an
    open binary file or a descriptor) at byte offset offset."""

    def __init__(self, f, width: int, height: int, opts: RawOptions = RawOptions(), offset: int = 0):
        _raw_size_check("NewRawSource", f, width, height)
        self.f, self.w, self.h, self.opts, self.offset = f, width, height, opts, offset

    def Size(self):
        return self.w, self.h

    def Masked(self) -> bool:
        return bool(self.opts.HasFill)

    def ReadWindow(self, dst: Float32Raster, x: int, y: int):
        import os

        if self.opts.HasFill and dst.valid is None:
            raise StrataPanic("engine: RawSource.ReadWindow: the source has a fill value and dst has no validity mask")
        fill = np.float32(self.opts.Fill)
        for row, k in _rows(dst, self.w):
            n = 4 * ((k - 1) * dst.stride + dst.width)
            b = os.pread(_fd(self.f), n, self.offset + 4 * ((y + row) * self.w + x))
            if len(b) < n:
                return SourceSinkError(f"engine: raw source: reading {_rows_name(y + row, k)}: unexpected EOF")
            cells = np.frombuffer(b, np.float32)
            s = row * dst.stride
            dst.data[s:s + cells.size] = cells
        if dst.valid is not None:
            for yy in range(dst.height):
                c = np.asarray(dst.data[yy * dst.stride:yy * dst.stride + dst.width])
                ok = ~np.isnan(c) if np.isnan(fill) else (c != fill) if self.opts.HasFill else np.ones(c.size, bool)
                _put_bits(dst.valid, dst.valid_offset + yy * dst.stride, ok.astype(np.uint8))
        return None


class RawSink(RasterSink):
    """engine.RawSink: writes a width×height raw float32 raster to f at
    byte offset offset, the fill value under invalid cells."""

    def __init__(self, f, width: int, height: int, opts: RawOptions = RawOptions(), offset: int = 0):
        _raw_size_check("NewRawSink", f, width, height)
        self.f, self.w, self.h, self.opts, self.offset = f, width, height, opts, offset

    def Size(self):
        return self.w, self.h

    def Masked(self) -> bool:
        return bool(self.opts.HasFill)

    def WriteWindow(self, src: Float32Raster, x: int, y: int):
        import os

        if src.valid is not None and not self.opts.HasFill:
            raise StrataPanic("engine: RawSink.WriteWindow: src has a validity mask and the sink has no fill value")
        fill = np.float32(self.opts.Fill)
        for row, k in _rows(src, self.w):
            n = (k - 1) * src.stride + src.width
            s = row * src.stride
            cells = np.array(src.data[s:s + n], np.float32)
            if src.valid is not None:
                for j in range(k):
                    bits = _bits(src.valid, src.valid_offset + (row + j) * src.stride, src.width)
                    seg = cells[j * src.stride:j * src.stride + src.width]
                    seg[bits == 0] = fill
            b = cells.tobytes()
            if os.pwrite(_fd(self.f), b, self.offset + 4 * ((y + row) * self.w + x)) < len(b):
                return SourceSinkError(f"engine: raw sink: writing {_rows_name(y + row, k)}: short write")
        return None


def process_raw(stages: StageList, dst: Sequence[RawSink], src: Sequence[RawSource],
                opts: Optional[Options] = None, ctx: Optional[Context] = None):
    """exec.ProcessChunked over raw files on the device (strata_process_raw).
    Returns None, Canceled, or a SourceSinkError."""
    dev = opts.Device if opts is not None else 0
    c = device_context(dev)

    def raw(r):
        f = _lib.RawFile()
        f.fd, f.has_fill, f.fill = _fd(r.f), 1 if r.opts.HasFill else 0, r.opts.Fill
        f.width, f.height, f.offset = r.w, r.h, r.offset
        return f

    srcs = (_lib.RawFile * len(src))(*[raw(s) for s in src])
    dsts = (_lib.RawFile * len(dst))(*[raw(d) for d in dst])
    o = c_opts(opts, ctx)
    cst = _lib.Stats()
    rc = _lib.lib().strata_process_raw(c, stages.c_array(), len(stages.stages), srcs, len(src), dsts, len(dst),
                                       ctypes.byref(o), ctypes.byref(cst))
    _stats_out(opts, cst)
    if rc == _lib.ECANCELED:
        return Canceled("context canceled")
    if rc == _lib.EIO:
        return SourceSinkError(_lib.last_error())
    _lib.check(rc)
    return None
