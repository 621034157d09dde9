"""The raster data model of strata (raster/raster.go, raster/window.go,
raster/mask.go), for callers of the device backend.

A Float32Raster is row-major float32 cells with a stride and an optional
LSB-first validity bitmap: cell (x, y) is ``data[y*stride + x]`` and its
validity bit ``valid_offset + y*stride + x`` of ``valid`` (set = valid,
``None`` = every cell valid). ``data`` is a 1-D numpy float32 array (host)
or a 1-D torch float32 CUDA tensor (device-resident); ``valid`` is a numpy
uint64 array or a torch int64 CUDA tensor of the same words.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Optional

import numpy as np


class StrataPanic(ValueError):
    """A programming error the reference reports with a panic; the message
    carries the reference's text and prefix ("terrain:", "engine:", ...)."""


class NotSupported(StrataPanic):
    """Valid for the reference, but not on the device backend (a caller
    would fall back to the CPU path)."""


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


@dataclass
class Float32Raster:
    data: Any
    width: int
    height: int
    stride: int
    valid: Optional[Any] = None
    valid_offset: int = 0

    # -- strata's accessors ---------------------------------------------
    def span(self) -> int:
        return (self.height - 1) * self.stride + self.width

    def on_device(self) -> bool:
        return _is_torch(self.data) and self.data.is_cuda

    def Row(self, y: int):
        if not 0 <= y < self.height:
            raise StrataPanic(f"raster: row {y} out of range [0, {self.height})")
        s = y * self.stride
        return self.data[s:s + self.width]

    def Index(self, x: int, y: int) -> int:
        if not (0 <= x < self.width and 0 <= y < self.height):
            raise StrataPanic(f"raster: cell ({x}, {y}) outside {self.width}×{self.height} raster")
        return y * self.stride + x

    def IsValid(self, x: int, y: int) -> bool:
        i = self.Index(x, y)
        return self.valid is None or MaskGet(self.valid, self.valid_offset + i)

    def SetValid(self, x: int, y: int, v: bool) -> None:
        i = self.Index(x, y)
        if self.valid is None:
            raise StrataPanic("raster: SetValid on a raster without a validity mask")
        MaskSet(self.valid, self.valid_offset + i, v)

    def Window(self, x: int, y: int, w: int, h: int) -> "Float32Raster":
        """A zero-copy view of the w×h cells at (x, y) (raster/window.go:12-33)."""
        if w <= 0 or h <= 0 or x < 0 or y < 0 or x + w > self.width or y + h > self.height:
            raise StrataPanic(
                f"raster: window {w}×{h} at ({x}, {y}) outside {self.width}×{self.height} raster")
        start = y * self.stride + x
        n = (h - 1) * self.stride + w
        return Float32Raster(self.data[start:start + n], w, h, self.stride, self.valid,
                             self.valid_offset + start)

    def Validate(self) -> None:
        if self.width <= 0 or self.height <= 0:
            raise StrataPanic(f"raster: dimensions must be positive, got {self.width}×{self.height}")
        if self.stride < self.width:
            raise StrataPanic(f"raster: stride {self.stride} is less than width {self.width}")
        n = self.span()
        if len(self.data) < n:
            raise StrataPanic(f"raster: data has {len(self.data)} cells, need {n}")
        if self.valid is not None:
            if self.valid_offset < 0:
                raise StrataPanic(f"raster: negative ValidOffset {self.valid_offset}")
            bits = len(self.valid) * 64
            if self.valid_offset > bits - n:
                raise StrataPanic(f"raster: mask has {bits} bits, need {self.valid_offset + n} "
                                  f"(offset {self.valid_offset} + {n} cells)")

    # -- conversions -----------------------------------------------------
    def numpy(self) -> np.ndarray:
        """The cells as a (height, width) float32 numpy array (a copy)."""
        d = self.data.detach().cpu().numpy() if _is_torch(self.data) else np.asarray(self.data)
        out = np.empty((self.height, self.width), np.float32)
        for y in range(self.height):
            out[y] = d[y * self.stride:y * self.stride + self.width]
        return out

    def valid_numpy(self) -> Optional[np.ndarray]:
        """The validity bits as a (height, width) bool array, or None."""
        if self.valid is None:
            return None
        v = self.valid.detach().cpu().numpy().view(np.uint64) if _is_torch(self.valid) else np.asarray(self.valid)
        bits = np.unpackbits(v.view(np.uint8), bitorder="little").astype(bool)
        out = np.empty((self.height, self.width), bool)
        for y in range(self.height):
            s = self.valid_offset + y * self.stride
            out[y] = bits[s:s + self.width]
        return out


def NewMask(n: int) -> np.ndarray:
    """A validity mask of n cells, every cell invalid (raster/mask.go)."""
    return np.zeros((n + 63) // 64, dtype=np.uint64)


def MaskWords(n: int) -> int:
    return (n + 63) // 64


def MaskGet(m, i: int) -> bool:
    return bool((int(m[i >> 6]) >> (i & 63)) & 1)


def MaskSet(m, i: int, v: bool) -> None:
    w = int(m[i >> 6])
    b = 1 << (i & 63)
    w = (w | b) if v else (w & ~b & 0xFFFFFFFFFFFFFFFF)
    m[i >> 6] = np.uint64(w)


def MaskFillRange(m, off: int, n: int, v: bool) -> None:
    for i in range(off, off + n):
        MaskSet(m, i, v)


def mask_from_bool(valid: np.ndarray, stride: Optional[int] = None, offset: int = 0,
                   words: Optional[int] = None) -> np.ndarray:
    """Packs a (height, width) bool array into LSB-first uint64 words with
    the given row stride and bit offset; bits outside the cells are 0."""
    h, w = valid.shape
    stride = w if stride is None else stride
    n = offset + (h - 1) * stride + w
    nwords = MaskWords(n) if words is None else words
    bits = np.zeros(nwords * 64, dtype=np.uint8)
    for y in range(h):
        s = offset + y * stride
        bits[s:s + w] = valid[y]
    return np.packbits(bits, bitorder="little").view(np.uint64).copy()


def NewFloat32(width: int, height: int, data) -> Float32Raster:
    return NewFloat32Stride(width, height, width, data)


def NewFloat32Stride(width: int, height: int, stride: int, data) -> Float32Raster:
    if width <= 0 or height <= 0:
        raise StrataPanic(f"raster: dimensions must be positive, got {width}×{height}")
    if stride < width:
        raise StrataPanic(f"raster: stride {stride} is less than width {width}")
    n = (height - 1) * stride + width
    if not _is_torch(data):
        data = np.ascontiguousarray(np.asarray(data, dtype=np.float32).reshape(-1))
    if len(data) < n:
        raise StrataPanic(f"raster: data has {len(data)} cells, need {n} for {width}×{height} with stride {stride}")
    return Float32Raster(data[:n], width, height, stride)


def NewFloat32Like(r: Float32Raster) -> Float32Raster:
    """A compact raster of r's size, zeroed, masked iff r is, in r's memory
    space (host numpy or device torch)."""
    n = r.width * r.height
    if r.on_device():
        import torch

        data = torch.zeros(n, dtype=torch.float32, device=r.data.device)
        valid = None
        if r.valid is not None:
            valid = torch.zeros(MaskWords(n), dtype=torch.int64, device=r.data.device)
        return Float32Raster(data, r.width, r.height, r.width, valid, 0)
    out = Float32Raster(np.zeros(n, np.float32), r.width, r.height, r.width)
    if r.valid is not None:
        out.valid = NewMask(n)
    return out
