"""Seeded synthetic rasters for tests and benchmarks.

The reference measures on synthetic fixtures of its own (splitmix64-based
FillDEM / RandomMask, benchmarks/internal/suite/suite.go:299-357); these
generators reuse splitmix64 for every random number and follow the
workloads' stated shapes and value distributions:

* fbm_dem: fractional-Brownian elevations by diamond-square (Hurst H),
  scaled to [lo, hi] metres;
* block_mask: a validity mask with a fraction of cells invalid as random
  non-overlapping 8x8 blocks;
* normal_trend: N(0, 1) (Box-Muller on splitmix64) plus a smooth trend;
* cell_mask: a validity mask with a fraction of random cells invalid.

Seeds are 0x5EED0000 + the workload number by default.
"""
from __future__ import annotations

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, start: int = 0) -> np.ndarray:
    """n consecutive outputs of splitmix64 from state seed (counter form)."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, n: int, start: int = 0) -> np.ndarray:
    """n uniforms in [0, 1) as float64 (the top 53 bits)."""
    return (splitmix64(seed, n, start) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def fbm_dem(width: int, height: int, seed: int, hurst: float = 0.8, lo: float = 0.0, hi: float = 3000.0) -> np.ndarray:
    """A (height, width) float32 fBm surface by diamond-square on the
    smallest 2^k + 1 lattice that covers it, cropped, scaled to [lo, hi]."""
    n = 1
    while n + 1 < max(width, height):
        n *= 2
    size = n + 1
    a = np.zeros((size, size), np.float32)
    ctr = 0

    def rnd(shape):
        nonlocal ctr
        k = int(np.prod(shape))
        u = uniform(seed, k, ctr).astype(np.float32).reshape(shape)
        ctr += k
        return u * np.float32(2) - np.float32(1)

    a[0::n, 0::n] = rnd((2, 2))
    step, scale = n, np.float32(1.0)
    decay = np.float32(2.0 ** -hurst)
    while step > 1:
        h = step // 2
        # Diamond: centres of squares.
        c = (a[0:-1:step, 0:-1:step] + a[0:-1:step, step::step] + a[step::step, 0:-1:step] + a[step::step, step::step])
        a[h::step, h::step] = c * np.float32(0.25) + rnd(c.shape) * scale
        # Square: edge midpoints, averaging the neighbours that exist.
        for r0, c0 in ((0, h), (h, 0)):
            rows = np.arange(r0, size, step)
            cols = np.arange(c0, size, step)
            s = np.zeros((rows.size, cols.size), np.float32)
            cnt = np.zeros((rows.size, cols.size), np.float32)
            for dr, dc in ((-h, 0), (h, 0), (0, -h), (0, h)):
                rr, cc = rows + dr, cols + dc
                okr = (rr >= 0) & (rr < size)
                okc = (cc >= 0) & (cc < size)
                sub = np.zeros((rows.size, cols.size), np.float32)
                sub[np.ix_(okr, okc)] = a[np.ix_(rr[okr], cc[okc])]
                s += sub
                cnt += np.outer(okr, okc).astype(np.float32)
            a[np.ix_(rows, cols)] = s / cnt + rnd(s.shape) * scale
        step = h
        scale = scale * decay
    a = a[:height, :width]
    mn, mx = float(a.min()), float(a.max())
    out = (a - np.float32(mn)) * np.float32((hi - lo) / (mx - mn if mx > mn else 1.0)) + np.float32(lo)
    return np.ascontiguousarray(np.clip(out, lo, hi), dtype=np.float32)


def block_mask(width: int, height: int, seed: int, fraction: float = 0.02, block: int = 8) -> np.ndarray:
    """(height, width) bool validity, with ceil(fraction*N/block^2) random
    block x block tiles of a block grid invalid (non-overlapping)."""
    valid = np.ones((height, width), bool)
    bx, by = (width + block - 1) // block, (height + block - 1) // block
    nb = int(np.ceil(fraction * width * height / (block * block)))
    nb = min(nb, bx * by)
    if nb == 0:
        return valid
    keys = splitmix64(seed ^ 0xB10C, bx * by)
    pick = np.argsort(keys, kind="stable")[:nb]
    for p in pick:
        y, x = divmod(int(p), bx)
        valid[y * block:(y + 1) * block, x * block:(x + 1) * block] = False
    return valid


def cell_mask(width: int, height: int, seed: int, fraction: float = 0.05) -> np.ndarray:
    """(height, width) bool validity with each cell invalid with probability fraction."""
    return uniform(seed ^ 0xCE11, width * height).reshape(height, width) >= fraction


def normal_trend(width: int, height: int, seed: int, trend: float = 0.001) -> np.ndarray:
    """(height, width) float32: N(0, 1) by Box-Muller on splitmix64, plus
    trend * (x + y)."""
    n = width * height
    u1 = uniform(seed, n)
    u2 = uniform(seed, n, n)
    z = np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)
    y, x = np.mgrid[0:height, 0:width]
    return (z.reshape(height, width) + trend * (x + y)).astype(np.float32)


def uniform_weights(n: int, seed: int) -> np.ndarray:
    """n float32 weights uniform in [-1, 1]."""
    return (uniform(seed ^ 0x3E16, n) * 2.0 - 1.0).astype(np.float32)
