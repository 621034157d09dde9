"""Float64 error of the float32 path - TEST INFRASTRUCTURE ONLY.

The device is bit-exact to the oracle (the C restatement of strata's
scalar kernels), so the oracle's distance from exact arithmetic is the
device's. This module restates each op's mathematics in float64 numpy
(the float32 inputs promoted exactly, the options' constants computed in
float64 from the options, no intermediate rounding to float32) and reports,
over the interior cells, the largest absolute difference and the
distribution of the difference in float32 ulps of the float64 value.

    python oracle/fp64_error.py [side]     # prints a markdown table

Formulas follow the reference (internal/stencil/horn.go:152-262,
aspect.go:97-173, curvature.go:79-129, rugged.go:70-103,
internal/focalrow/focalrow.go:217-315, internal/curve/scalar.go:39-114).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if sys.path and os.path.abspath(sys.path[0]) == HERE:
    sys.path[0] = ROOT  # run as a script: import the oracle package, not this folder's module
elif ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402


def _win(a, r):
    """(h - 2r, w - 2r, 2r+1, 2r+1) windows of a float64 array."""
    return np.lib.stride_tricks.sliding_window_view(a, (2 * r + 1, 2 * r + 1))


def _run(stages, cells):
    h, w = cells.shape
    src = dict(data=np.ascontiguousarray(cells.reshape(-1)), width=w, height=h, stride=w, valid=None,
               valid_offset=0)
    out = dict(data=np.zeros(w * h, np.float32), width=w, height=h, stride=w, valid=None, valid_offset=0)
    orc.process(stages, src, [out], nthreads=os.cpu_count() or 1)
    return out["data"].reshape(h, w)


def _ulps(got, want):
    """|got - want| in float32 ulps of want (ulps of the smallest normal below it)."""
    a = np.abs(want)
    e = np.floor(np.log2(np.maximum(a, 2.0 ** -126)))
    return np.abs(got.astype(np.float64) - want) / 2.0 ** (e - 23)


def _horn(z, cs):
    w = _win(z, 1)
    z1, z2, z3 = w[..., 0, 0], w[..., 0, 1], w[..., 0, 2]
    z4, z6 = w[..., 1, 0], w[..., 1, 2]
    z7, z8, z9 = w[..., 2, 0], w[..., 2, 1], w[..., 2, 2]
    dx = ((z3 - z1) + (z9 - z7)) + 2 * (z6 - z4)
    dy = ((z7 - z1) + (z9 - z3)) + 2 * (z8 - z2)
    return dx / (8 * cs), dy / (8 * cs)


def report(side=512, seed=0x5EED0002):
    from strata_b200 import synth  # the generator only; no device code runs

    dem = synth.fbm_dem(side, side, seed)
    foc = synth.normal_trend(side, side, seed)
    z = dem.astype(np.float64)
    f = foc.astype(np.float64)
    cs = 10.0
    rows = []

    def add(name, got, want, r, circular=False):
        g = got[r:-r, r:-r]
        ok = np.isfinite(g) & np.isfinite(want)
        d = np.abs(g[ok].astype(np.float64) - want[ok])
        if circular:
            d = np.minimum(d, 360.0 - d)
        u = _ulps(g[ok], want[ok]) if not circular else d / 2.0 ** (np.floor(np.log2(np.maximum(np.abs(want[ok]), 1.0))) - 23)
        rows.append(dict(op=name, cells=int(ok.sum()), max_abs=float(d.max()), p50_ulp=float(np.percentile(u, 50)),
                         p99_ulp=float(np.percentile(u, 99)), max_ulp=float(u.max())))

    kx, ky = orc.horn_scales(cs, cs, 1.0)
    gx, gy = _horn(z, cs)
    m = np.hypot(gx, gy)
    # Slope in degrees: Atan32(magnitude) x 180/pi.
    st = orc.stage(orc.SLOPE, 1, 1, k=(kx, ky, np.float32(180 / math.pi)))
    add("slope (degrees)", _run([st], dem), np.degrees(np.arctan(m)), 1)
    # Aspect (compass): atan2(-gx, gy) in degrees, folded into [0, 360).
    st = orc.stage(orc.ASPECT, 1, 0, k=(kx, ky, -1.0))
    a = np.degrees(np.arctan2(-gx, gy))
    a = np.where(a < 0, a + 360, a)
    add("aspect", _run([st], dem), a, 1, circular=True)
    # Hillshade, azimuth 315, altitude 45.
    c3 = orc.hillshade_light(315.0, 45.0)
    alt, az = math.radians(45.0), math.radians(315.0)
    c, bx, by = 255 * math.sin(alt), -255 * math.cos(alt) * math.sin(az), 255 * math.cos(alt) * math.cos(az)
    st = orc.stage(orc.HILLSHADE, 1, 0, k=(kx, ky, *c3))
    hs = np.clip((c + bx * gx + by * gy) / np.sqrt(1 + gx * gx + gy * gy), 0, 255)
    add("hillshade", _run([st], dem), hs, 1)
    # Zevenbergen-Thorne curvature.
    k5 = orc.zt_scales(cs, cs, 1.0)
    w = _win(z, 1)
    P = (w[..., 1, 2] - w[..., 1, 0]) / (2 * cs)
    Q = (w[..., 2, 1] - w[..., 0, 1]) / (2 * cs)
    R = (w[..., 1, 0] + w[..., 1, 2] - 2 * w[..., 1, 1]) / cs ** 2
    T = (w[..., 0, 1] + w[..., 2, 1] - 2 * w[..., 1, 1]) / cs ** 2
    S = (w[..., 0, 0] + w[..., 2, 2] - w[..., 0, 2] - w[..., 2, 0]) / (4 * cs * cs)
    p2, q2, pq = P * P, Q * Q, P * Q
    g = p2 + q2
    with np.errstate(divide="ignore", invalid="ignore"):
        prof = -(p2 * R + 2 * pq * S + q2 * T) / g / (1 + g) ** 1.5
        plan = -(q2 * R - 2 * pq * S + p2 * T) / g / np.sqrt(g)
    mean = -((1 + q2) * R - 2 * pq * S + (1 + p2) * T) / (2 * (1 + g) ** 1.5)
    for kind, name, want in ((0, "curvature profile", prof), (1, "curvature plan", plan), (2, "curvature mean", mean)):
        add(name, _run([orc.stage(orc.CURVATURE, 1, kind, k=k5)], dem), want, 1)
    # Ruggedness at r = 1.
    c0 = w[..., 1, 1]
    nb = w.reshape(w.shape[0], w.shape[1], 9)
    add("TRI (Riley)", _run([orc.stage(orc.RUGGEDNESS, 1, 0)], dem), np.sqrt(((nb - c0[..., None]) ** 2).sum(-1)), 1)
    add("TPI", _run([orc.stage(orc.RUGGEDNESS, 1, 2)], dem), c0 - (nb.sum(-1) - c0) / 8, 1)
    add("roughness", _run([orc.stage(orc.RUGGEDNESS, 1, 3)], dem), nb.max(-1) - nb.min(-1), 1)
    # Focal ops.
    for r in (3, 8):
        wts = synth.uniform_weights((2 * r + 1) ** 2, 0x5EED0003 + r)
        wf = _win(f, r)
        want = (wf * wts.astype(np.float64).reshape(2 * r + 1, 2 * r + 1)).sum((-1, -2))
        add(f"correlate r{r}", _run([orc.stage(orc.CORRELATE, r, 0, tables=(wts,))], foc), want, r)
        add(f"mean r{r}", _run([orc.stage(orc.MEAN, r)], foc), wf.mean((-1, -2)), r)
        add(f"max r{r}", _run([orc.stage(orc.MAX, r)], foc), wf.max((-1, -2)), r)
    taps = orc.gaussian(8, 2.5)
    t = taps.astype(np.float64)
    want = np.einsum("ijab,a,b->ij", _win(f, 8), t, t)
    add("gaussian r8", _run([orc.stage(orc.SEPARABLE, 8, 0, tables=(taps, taps))], foc), want, 8)
    return rows


def markdown(rows):
    out = ["| op | interior cells | max abs error | p50 ulps | p99 ulps | max ulps |", "|---|---:|---:|---:|---:|---:|"]
    for r in rows:
        out.append(f"| {r['op']} | {r['cells']} | {r['max_abs']:.3g} | {r['p50_ulp']:.2f} | {r['p99_ulp']:.2f} | "
                   f"{r['max_ulp']:.3g} |")
    return "\n".join(out)


if __name__ == "__main__":
    print(markdown(report(int(sys.argv[1]) if len(sys.argv) > 1 else 512)))
