"""Python binding of the parity oracle - TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the C restatement of strata's scalar kernels in
strata_oracle.c) through ctypes. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs import this module; the product never does.

Rasters are described by plain numpy arrays: ``data`` is a 1-D float32
array holding (height-1)*stride + width cells, ``valid`` an optional 1-D
uint64 array of LSB-first validity bits starting at bit ``valid_offset``
(strata's raster.Float32Raster layout, raster/raster.go:41-54).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

GRADIENT, SLOPE, ASPECT, HILLSHADE, CURVATURE, RUGGEDNESS = 1, 2, 3, 4, 5, 6
CORRELATE, SEPARABLE, MEAN, MIN, MAX, LOOKUP, RECLASS = 7, 8, 9, 10, 11, 12, 13
HEATLOAD, ORIENTATION, STEP = 14, 15, 16
# vec.Op (internal/vec/chain.go:24-38): the kind of a STEP stage
(VEC_ADD, VEC_SUB, VEC_MUL, VEC_DIV, VEC_MIN, VEC_MAX, VEC_ADD_SCALAR, VEC_MUL_SCALAR, VEC_AFFINE, VEC_SUB_DIV,
 VEC_CLAMP, VEC_ABS, VEC_SQRT) = range(13)
STAGE_FIT = 2  # the derivatives from Wood's quadratic fit over the (2 radius + 1)^2 window


class Stage(ctypes.Structure):
    _fields_ = [
        ("op", ctypes.c_uint32),
        ("radius", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("k", ctypes.c_float * 16),
        ("table", ctypes.c_void_p * 4),
        ("table_len", ctypes.c_int32 * 4),
        ("input", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class Raster(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("width", ctypes.c_int64),
        ("height", ctypes.c_int64),
        ("stride", ctypes.c_int64),
        ("valid", ctypes.c_void_p),
        ("valid_offset", ctypes.c_int64),
    ]


def build() -> str:
    """Compiles liboracle.so from strata_oracle.c (make, in this folder)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "strata_oracle.c")
        if not os.path.exists(LIB_PATH) or (
            os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(LIB_PATH)
        ):
            build()
        L = ctypes.CDLL(LIB_PATH)
        f, d, i64, p = ctypes.c_float, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p
        L.orc_atan32.restype = f
        L.orc_atan32.argtypes = [f]
        L.orc_atan2f32.restype = f
        L.orc_atan2f32.argtypes = [f, f]
        L.orc_go_min.restype = f
        L.orc_go_min.argtypes = [f, f]
        L.orc_go_max.restype = f
        L.orc_go_max.argtypes = [f, f]
        L.orc_atan32_array.argtypes = [p, p, i64]
        L.orc_atan32_drops.restype = i64
        L.orc_atan32_drops.argtypes = [ctypes.c_int]
        L.orc_atan2f32_array.argtypes = [p, p, p, i64]
        L.orc_horn_scales.argtypes = [d, d, d, ctypes.POINTER(f), ctypes.POINTER(f)]
        L.orc_zt_scales.argtypes = [d, d, d, ctypes.POINTER(f)]
        L.orc_hillshade_light.argtypes = [d, d, ctypes.POINTER(f)]
        L.orc_gaussian.argtypes = [ctypes.c_int, d, ctypes.POINTER(f)]
        L.orc_process.restype = ctypes.c_int
        L.orc_process.argtypes = [ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(Raster),
                                  ctypes.POINTER(Raster), ctypes.c_int, ctypes.c_int]
        L.orc_process_ex.restype = ctypes.c_int
        L.orc_process_ex.argtypes = [ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(Raster),
                                     ctypes.POINTER(Raster), ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_process_n.restype = ctypes.c_int
        L.orc_process_n.argtypes = [ctypes.POINTER(Stage), ctypes.c_int, ctypes.POINTER(Raster), ctypes.c_int,
                                    ctypes.POINTER(Raster), ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


# ---------------------------------------------------------------------------
# Scalar helpers.

def atan32(x: float) -> np.float32:
    return np.float32(lib().orc_atan32(np.float32(x)))


def atan2f32(y: float, x: float) -> np.float32:
    return np.float32(lib().orc_atan2f32(np.float32(y), np.float32(x)))


def atan32_array(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    lib().orc_atan32_array(x.ctypes.data, out.ctypes.data, x.size)
    return out


def atan32_drops(nthreads: int) -> int:
    """Arguments among all 2^31 non-negative floats where Atan32 falls."""
    return int(lib().orc_atan32_drops(nthreads))


def atan2f32_array(y: np.ndarray, x: np.ndarray) -> np.ndarray:
    y = np.ascontiguousarray(y, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(y)
    lib().orc_atan2f32_array(y.ctypes.data, x.ctypes.data, out.ctypes.data, y.size)
    return out


def go_min(a, b):
    return np.float32(lib().orc_go_min(np.float32(a), np.float32(b)))


def go_max(a, b):
    return np.float32(lib().orc_go_max(np.float32(a), np.float32(b)))


def horn_scales(cx, cy, z):
    kx, ky = ctypes.c_float(), ctypes.c_float()
    lib().orc_horn_scales(cx, cy, z, ctypes.byref(kx), ctypes.byref(ky))
    return np.float32(kx.value), np.float32(ky.value)


def zt_scales(cx, cy, z):
    out = (ctypes.c_float * 5)()
    lib().orc_zt_scales(cx, cy, z, out)
    return [np.float32(v) for v in out]


def hillshade_light(azimuth, altitude):
    out = (ctypes.c_float * 3)()
    lib().orc_hillshade_light(azimuth, altitude, out)
    return [np.float32(v) for v in out]


def gaussian(radius, sigma):
    out = (ctypes.c_float * (2 * radius + 1))()
    lib().orc_gaussian(radius, sigma, out)
    return np.array(list(out), dtype=np.float32)


# ---------------------------------------------------------------------------
# Whole-raster calls.

def stage(op, radius=0, kind=0, k=(), tables=(), flags=0, input=-1):
    """Builds a Stage; returns (stage, keepalive) so table arrays outlive it."""
    st = Stage()
    st.op, st.radius, st.kind, st.flags, st.input = op, radius, kind, flags, input
    for i, v in enumerate(k):
        st.k[i] = float(v)
    keep = []
    for i, t in enumerate(tables):
        a = np.ascontiguousarray(t, dtype=np.float32)
        keep.append(a)
        st.table[i] = a.ctypes.data
        st.table_len[i] = a.size
    return st, keep


def _raster(data, width, height, stride, valid=None, valid_offset=0):
    r = Raster()
    r.data = data.ctypes.data
    r.width, r.height, r.stride = width, height, stride
    r.valid = valid.ctypes.data if valid is not None else None
    r.valid_offset = valid_offset
    return r


def process(stages, src, dsts, nthreads=1, simd=False):
    """Runs stages over src into dsts.

    stages: list of (Stage, keepalive) from stage().
    src, dsts[i]: dicts with keys data, width, height, stride, valid, valid_offset.
    simd: run the radius-1 stencils through the restated AVX2 lanes
    (strata_avx2.c, the reference's AVX2 path; the same bits).
    """
    st_arr = (Stage * len(stages))(*[s for s, _ in stages])
    s = _raster(**src)
    d_arr = (Raster * len(dsts))(*[_raster(**d) for d in dsts])
    rc = lib().orc_process_ex(st_arr, len(stages), ctypes.byref(s), d_arr, len(dsts), nthreads, 1 if simd else 0)
    if rc != 0:
        raise ValueError(f"oracle: invalid call (rc={rc})")


def process_n(stages, srcs, dsts, nthreads=1):
    """Runs a pipeline over several inputs (a pointwise chain whose binary
    steps read srcs[input]); srcs and dsts as process() takes them."""
    st_arr = (Stage * len(stages))(*[s for s, _ in stages])
    s_arr = (Raster * len(srcs))(*[_raster(**x) for x in srcs])
    d_arr = (Raster * len(dsts))(*[_raster(**d) for d in dsts])
    rc = lib().orc_process_n(st_arr, len(stages), s_arr, len(srcs), d_arr, len(dsts), nthreads)
    if rc != 0:
        raise ValueError(f"oracle: invalid call (rc={rc})")


def step_stage(op, input=-1, k0=0.0, k1=0.0):
    """One vec.Chain step (kind = the vec.Op)."""
    return stage(STEP, 0, op, (k0, k1), input=input)


def rescale_range_coeffs(in_lo, in_hi, out_lo, out_hi):
    """transfer.rescaleCoeffs (transfer/transfer.go:236-250) without its
    checks: a = f32((outHi - outLo) / (inHi - inLo)), b = f32(outLo - a*inLo)
    in float64."""
    a = np.float32((float(np.float32(out_hi)) - float(np.float32(out_lo))) /
                   (float(np.float32(in_hi)) - float(np.float32(in_lo))))
    b = np.float32(float(np.float32(out_lo)) - float(a) * float(np.float32(in_lo)))
    return a, b


# ---------------------------------------------------------------------------
# Stages from the terrain, focal and transfer options, resolved as the
# reference's option code resolves them (terrain/stencil.go:16-49,
# slope.go:84-95, aspect.go:97-102, hillshade.go:94-117, curvature.go:
# 113-127, ruggedness.go:119-141, transfer/transfer.go:184-212), for
# callers that must not load the device library (the benchmark's
# reference arm). Defaults: cell size 1, z factor 1.

def _cells(cell_size, cell_size_y, z_factor):
    cx = cell_size or 1.0
    cy = cell_size_y or cx
    return cx, cy, (z_factor or 1.0)


def gradient_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0):
    kx, ky = horn_scales(*_cells(cell_size, cell_size_y, z_factor))
    return stage(GRADIENT, 1, 0, [kx, ky])


def slope_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0, units=0):
    """units: 0 degrees, 1 percent, 2 radians (terrain.SlopeUnits)."""
    kx, ky = horn_scales(*_cells(cell_size, cell_size_y, z_factor))
    scale, take_atan = {0: (np.float32(180 / np.pi), 1), 1: (np.float32(100), 0), 2: (np.float32(1), 1)}[units]
    return stage(SLOPE, 1, take_atan, [kx, ky, scale])


def aspect_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0, zero_for_flat=False, trigonometric=False):
    kx, ky = horn_scales(*_cells(cell_size, cell_size_y, z_factor))
    return stage(ASPECT, 1, 1 if trigonometric else 0, [kx, ky, 0.0 if zero_for_flat else -1.0])


def hillshade_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0, azimuth=315.0, altitude=45.0):
    kx, ky = horn_scales(*_cells(cell_size, cell_size_y, z_factor))
    c, bx, by = hillshade_light(azimuth, altitude)
    return stage(HILLSHADE, 1, 0, [kx, ky, c, bx, by])


def curvature_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0, kind=0):
    return stage(CURVATURE, 1, kind, zt_scales(*_cells(cell_size, cell_size_y, z_factor)))


def ruggedness_stage(kind=0, radius=1):
    return stage(RUGGEDNESS, radius, kind)


def lookup_stage(xs, ys):
    return stage(LOOKUP, 0, 0, (), [np.asarray(xs, np.float32), np.asarray(ys, np.float32)])


def reclass_stage(breaks, values):
    return stage(RECLASS, 0, 0, (), [np.asarray(breaks, np.float32), np.asarray(values, np.float32)])


def pack_mask(valid: np.ndarray) -> np.ndarray:
    """A (h, w) bool validity mask as LSB-first 64-bit words, row-major with
    stride w (raster/mask.go's layout)."""
    bits = np.packbits(np.asarray(valid, bool).reshape(-1), bitorder="little")
    pad = (-bits.size) % 8
    if pad:
        bits = np.concatenate([bits, np.zeros(pad, np.uint8)])
    return bits.view(np.uint64).copy()


# McCune and Keon's regressions (terrain/heatload.go:104-108): K0, the
# cos(S) coefficient, the cos(A')sin(S) and sin(S) latitude terms, the
# folded term and Equation 3's constant.
HEATLOAD_COEFFICIENTS = [
    (-1.467, 1.582, -1.500, -0.262, 0.607, 0.0),
    (-1.236, 1.350, -1.376, -0.331, 0.375, 0.0),
    (0.339, 0.808, 0.0, -0.196, 0.0, -0.482),
]


def heatload_terms(latitude, equation=0, radiation=False, linear=False):
    """heatLoadTerms (terrain/heatload.go:110-142): K0, A, BX, BY, E, F, CX,
    CY in float64, and whether exp is taken."""
    import math

    k = HEATLOAD_COEFFICIENTS[equation]
    lat = abs(latitude) * math.pi / 180
    sin_l, cos_l = math.sin(lat), math.cos(lat)
    h = math.sqrt(2) / 2
    cos_c, sin_c = h, h
    south = latitude < 0
    if radiation and not south:
        cos_c, sin_c = 1.0, 0.0
    elif radiation and south:
        cos_c, sin_c = -1.0, 0.0
    elif south:
        cos_c, sin_c = -h, h
    kc = k[2] * sin_l + k[5]
    terms = [k[0], k[1] * cos_l, -kc * sin_c, kc * cos_c, k[3] * sin_l, k[4], cos_c, sin_c]
    return np.array(terms, np.float64), bool(linear and equation != 2)


def fit_scales(fit_radius, cx, cy, z):
    """newWoodFit's factors kp, kq, kr, kt, ks (terrain/fit.go:38-60), each
    computed in float64 and rounded once."""
    r = fit_radius
    q = float(sum((3 * i * i - r * (r + 1)) ** 2 for i in range(-r, r + 1)))
    k = float(2 * r + 1)
    s = float(r * (r + 1) * (2 * r + 1)) / 3
    return [np.float32(z / (k * s * cx)), np.float32(z / (k * s * cy)), np.float32(6 * z / (k * q * cx * cx)),
            np.float32(6 * z / (k * q * cy * cy)), np.float32(z / (s * s * cx * cy))]


def heatload_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0, latitude=45.0, equation=0, radiation=False,
                   linear=False, fit_radius=0):
    terms, ex = heatload_terms(latitude, equation, radiation, linear)
    table = terms.view(np.float32)
    cx, cy, z = _cells(cell_size, cell_size_y, z_factor)
    if fit_radius:
        return stage(HEATLOAD, fit_radius, int(ex), fit_scales(fit_radius, cx, cy, z), [table], STAGE_FIT)
    kx, ky = horn_scales(cx, cy, z)
    return stage(HEATLOAD, 1, int(ex), [kx, ky], [table])


def orientation_stage(cell_size=1.0, cell_size_y=0.0, z_factor=1.0, east=False, unweighted=False, fit_radius=0):
    kind = (1 if east else 0) | (2 if unweighted else 0)
    cx, cy, z = _cells(cell_size, cell_size_y, z_factor)
    if fit_radius:
        return stage(ORIENTATION, fit_radius, kind, fit_scales(fit_radius, cx, cy, z), [], STAGE_FIT)
    kx, ky = horn_scales(cx, cy, z)
    return stage(ORIENTATION, 1, kind, [kx, ky])


def fit_stage(op, fit_radius, cell_size=1.0, cell_size_y=0.0, z_factor=1.0, kind=0, consts=()):
    """A product of Wood's fit: op GRADIENT, SLOPE (consts: scale; kind: take
    the arctangent), ASPECT (flat; kind: trigonometric), HILLSHADE (c, bx,
    by) or CURVATURE (kind)."""
    cx, cy, z = _cells(cell_size, cell_size_y, z_factor)
    return stage(op, fit_radius, kind, fit_scales(fit_radius, cx, cy, z) + list(consts), [], STAGE_FIT)
