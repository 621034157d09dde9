"""Writes tests/golden/kat.json: the known-answer vectors of strata's own
tests for the raster-stencil path, transcribed from the reference's test
sources (cited per case, paths within the strata project). Every float is
stored as its float32 bit pattern so the fixture is exact.

    python tests/golden/make_kat.py

The reference is Go and no Go toolchain exists here, so nothing is
executed: these are the expected values the reference's tests assert.
"""
from __future__ import annotations

import json
import math
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))

NAN = float("nan")
INF = float("inf")
NZ = -0.0


def b(x: float) -> str:
    """float32 bits of x as hex."""
    return "0x%08x" % struct.unpack("<I", struct.pack("<f", x))[0]


def f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", x))[0]


def bits(xs):
    return [b(x) for x in xs]


PI32 = f32(math.pi)

cases = {}

# internal/stencil/stencil_test.go:386-410 (TestAtan2F32Accuracy's table):
# exact expected bits.
cases["atan2f32_exact"] = {
    "cite": "internal/stencil/stencil_test.go:386-410",
    "rows": [[b(y), b(x), b(w)] for y, x, w in [
        (0, 0, 0),
        (NZ, 0, NZ),
        (0, NZ, PI32),
        (NZ, NZ, -PI32),
        (0, -5, PI32),
        (NZ, -5, -PI32),
        (5, 0, f32(PI32 / 2)),
        (-5, NZ, -f32(PI32 / 2)),
        (INF, INF, f32(PI32 / 4)),
        (-INF, -INF, -f32(PI32 - f32(PI32 / 4))),
        (3, -INF, PI32),
        (-INF, 3, -f32(PI32 / 2)),
    ]],
}

# internal/stencil/stencil_test.go:35-43: Atan32's special values.
cases["atan32_exact"] = {
    "cite": "internal/stencil/stencil_test.go:35-43",
    "rows": [[b(0.0), b(0.0)], [b(INF), b(f32(math.pi / 2))]],
    "nan_in_nan_out": True,
}

# internal/stencil/stencil_test.go:326-329: atan2Specials.
cases["atan2_specials"] = {
    "cite": "internal/stencil/stencil_test.go:326-329",
    "values": bits([0, NZ, INF, -INF, NAN, 1, -1, 0.5, -2, 3e38, -3e38, 1.401298464324817e-45,
                    -1.401298464324817e-45, 1e-30, -7e20]),
    "bound": 3e-7,
}

# internal/stencil/stencil_test.go:458-484 (TestRuggednessRowKnownWindows):
# exact bits for Riley, Wilson, TPI and roughness.
tiny = math.ldexp(1, -12)
cases["ruggedness_windows"] = {
    "cite": "internal/stencil/stencil_test.go:458-484",
    "rows": [
        {"name": "flat", "w": bits([7] * 9), "want": bits([0, 0, 0, 0])},
        {"name": "3-4-5", "w": bits([3, 4, 0, 0, 0, 0, 0, 0, 0]), "want": bits([5, 0.875, -0.875, 4])},
        {"name": "pit", "w": bits([2, 2, 2, 2, -6, 2, 2, 2, 2]), "want": bits([f32(math.sqrt(512)), 8, -8, 8])},
        {"name": "spread", "w": bits([-1, 5, 2, 0, 3, -4, 1, 1, 9]),
         "want": bits([f32(math.sqrt(16 + 4 + 1 + 9 + 49 + 4 + 4 + 36)), 3.375, 3 - 1.625, 13])},
        {"name": "float64 sum", "w": bits([1, tiny, tiny, tiny, 0, tiny, tiny, tiny, tiny]),
         "want": bits([f32(1 + math.ldexp(1, -22)), f32(f32(1 + 7 * tiny) * 0.125),
                       f32(-f32(1 + 7 * tiny) * 0.125), 1])},
    ],
}

# internal/stencil/stencil_test.go:486-497 (TestRoughnessNaNAndSignedZero).
cases["roughness_special"] = {
    "cite": "internal/stencil/stencil_test.go:486-497",
    "nan_window": bits([1, 2, 3, 4, NAN, 6, 7, 8, 9]),
    "zero_window": bits([0, NZ, 0, NZ, 0, 0, 0, 0, NZ]),
    "zero_want": b(0.0),
}

# terrain/terrain_test.go:126-159 (TestHandComputed, Esri's slope example).
cases["slope_esri"] = {
    "cite": "terrain/terrain_test.go:126-159",
    "dem": bits([50, 45, 50, 30, 30, 30, 8, 10, 10]),
    "cell_size": 5,
    "dx": 0.05, "dy": -3.8, "grad_tol": 1e-6,
    "units": [[0, 75.25762, 1e-4], [1, 100 * math.hypot(0.05, 3.8), 1e-3], [2, math.atan(math.hypot(0.05, 3.8)), 1e-6]],
}

# terrain/shade_test.go:145-160 (TestAspectHandComputed).
cases["aspect_esri"] = {
    "cite": "terrain/shade_test.go:145-160",
    "dem": bits([101, 92, 85, 101, 92, 85, 101, 91, 84]),
    "cell_size": 5,
    "want": 90 + math.atan(0.375 / 8.125) * 180 / math.pi,
    "tol": 1e-4,
}

# terrain/shade_test.go:288-303 (TestHillshadeHandComputed).
_s = math.atan(math.hypot(1.625, 0.075))
_asp = (90 + math.atan(0.075 / 1.625) * 180 / math.pi) * math.pi / 180
cases["hillshade_esri"] = {
    "cite": "terrain/shade_test.go:288-303",
    "dem": bits([101, 92, 85, 101, 92, 85, 101, 91, 84]),
    "cell_size": 5,
    "default_light_want": b(0.0),
    "azimuth_90_want": 255 * (math.sin(math.pi / 4) * math.cos(_s) + math.cos(math.pi / 4) * math.sin(_s)
                              * math.cos(math.pi / 2 - _asp)),
    "tol": 1e-3,
}

# terrain/curvature_test.go:232-260 (TestCurvatureHandComputed).
cases["curvature_hand"] = {
    "cite": "terrain/curvature_test.go:232-260",
    "dem": bits([10, 12, 15, 11, 13, 17, 13, 16, 20]),
    "want": [[0, -32 / (13 * 14 ** 1.5)], [1, -20 / 13 ** 1.5], [2, -12 / 14 ** 1.5]],
    "rel_tol": 1e-6,
}

# focal/focal_test.go:163-203 (TestHandComputed): src(x, y) = 10y + x.
cases["focal_hand"] = {
    "cite": "focal/focal_test.go:163-203",
    "src": bits([0, 1, 2, 10, 11, 12, 20, 21, 22]),
    "weights": bits([0, 0, 1, 0, 0, 0, 0, 0, 0]),
    "correlate": b(2), "convolve": b(20),
    "separable_shift": {"row": bits([0, 0, 1]), "col": bits([1, 0, 0]), "want": b(2)},
    "separable_sums": {"row": bits([1, 1, 1]), "col": bits([1, 2, 1]),
                       "want": b(0 + 1 + 2 + 2 * (10 + 11 + 12) + 20 + 21 + 22)},
    "mean": b(11), "min": b(0), "max": b(22),
}

# internal/curve/curve_test.go:34-91 (TestReclass).
cases["reclass"] = {
    "cite": "internal/curve/curve_test.go:34-91",
    "rows": [
        {"breaks": bits([10, 20, 30]), "values": bits([1, 2, 3, 4]),
         "src": bits([9.999, 10, 10.001, 19.999, 20, 29.999, 30, 30.001]), "want": bits([1, 2, 2, 2, 3, 3, 4, 4])},
        {"breaks": bits([0]), "values": bits([-1, 1]),
         "src": bits([-INF, -3.4028234663852886e38, -0.001, 0, 0.001, 3.4028234663852886e38, INF]),
         "want": bits([-1, -1, -1, 1, 1, 1, 1])},
        {"breaks": bits([0]), "values": bits([7, 8]), "src": bits([NZ, 0]), "want": bits([8, 8])},
        {"breaks": bits([10, 20]), "values": bits([1, 2, 3]), "src": bits([NAN, 15]), "want": bits([NAN, 2])},
        {"breaks": [], "values": bits([5]), "src": bits([-1, 0, 1, INF, -INF]), "want": bits([5, 5, 5, 5, 5])},
        {"breaks": bits([1, 2]), "values": bits([NAN, INF, NZ]), "src": bits([0, 1.5, 3]),
         "want": bits([NAN, INF, NZ])},
    ],
}

# internal/curve/curve_test.go:102-186 (TestLookup).
cases["lookup"] = {
    "cite": "internal/curve/curve_test.go:102-186",
    "rows": [
        {"xs": bits([0, 10, 20]), "ys": bits([0, 1, 0]), "src": bits([-5, 0, 2.5, 5, 10, 15, 20, 25]),
         "want": bits([0, 0, 0.25, 0.5, 1, 0.5, 0, 0])},
        {"xs": bits([-3, 0.1, 7.25, 1000]), "ys": bits([5, -2.5, 0.125, 1e30]), "src": bits([-3, 0.1, 7.25, 1000]),
         "want": bits([5, -2.5, 0.125, 1e30])},
        {"xs": bits([0, 1, 2, 3, 4]), "ys": bits([10, NAN, INF, NZ, 20]), "src": bits([0, 1, 2, 3, 4]),
         "want": bits([10, NAN, INF, NZ, 20])},
        {"xs": bits([0, 1, 2]), "ys": bits([10, NAN, 20]), "src": bits([0.5, 1.5]), "want": bits([NAN, NAN])},
        {"xs": bits([4]), "ys": bits([9]), "src": bits([-1, 4, 100, INF, -INF]), "want": bits([9, 9, 9, 9, 9])},
        {"xs": bits([0, 1]), "ys": bits([-2, 3]), "src": bits([-INF, INF]), "want": bits([-2, 3])},
        {"xs": bits([0, 1]), "ys": bits([-2, 3]), "src": bits([NAN, 0.5]), "want": bits([NAN, 0.5])},
        {"xs": bits([0, 10]), "ys": bits([2, 2]), "src": bits([0, 3, 7, 10]), "want": bits([2, 2, 2, 2])},
        {"xs": bits([0, 1, 2]), "ys": bits([0, 10, 20]), "src": bits([1]), "want": bits([10])},
    ],
}

# internal/curve/curve_test.go:188-212 (TestLookupIsNotFused): the cell
# just below 1 with ys (-1, 2^-23) must give +0 (product rounded, then
# added), not the fused 2^-24 - 2^-47.
cases["lookup_not_fused"] = {
    "cite": "internal/curve/curve_test.go:188-212",
    "xs": bits([0, 1]), "ys": bits([-1, math.ldexp(1, -23)]),
    "src": "0x3f7fffff", "want": b(0.0),
}

# transfer/transfer_test.go:420-438 (TestKnotsAreExact).
cases["knots_exact"] = {
    "cite": "transfer/transfer_test.go:420-438",
    "xs": bits([-3, 0, 7.25, 1000, 2000]), "ys": bits([5, NAN, INF, NZ, 20]),
}

# internal/curve/curve_test.go:93-100 (TestReclassNaNPayload): a NaN cell
# comes back as itself.
cases["nan_payload"] = {
    "cite": "internal/curve/curve_test.go:93-100",
    "src": ["0x7fc00001", "0xffc00000"],
}

# terrain/heatload_test.go:15-47 (mcCuneKeonTest, TestHeatLoadMcCuneKeon,
# :66-109): McCune and Keon's spreadsheet, latitude, slope and aspect in
# degrees, then Equations 1-3 for radiation and for heat load, each as the
# equation gives it (ln for 1 and 2), held to 2e-6 on a 5x5 plane on unit
# cells (z = +-tan(slope) * row).
cases["heatload_mccune_keon"] = {
    "cite": "terrain/heatload_test.go:15-47,66-109",
    "tol": 2e-6,
    "rows": [
        [40, 0, 0, [-0.25511769098577686, -0.20184000178937955, 0.9579639100401343],
         [-0.25511769098577686, -0.20184000178937955, 0.9579639100401343]],
        [40, 30, 0, [-0.9837750181305804, -0.8890103948393941, 0.5710452843712215],
         [-0.6279670110295916, -0.6268993985409437, 0.6416325501052635]],
        [40, 30, 180, [-0.01959360360077163, -0.00453464391071629, 1.0530452843712215],
         [0.053812205478473735, -0.001480597264211625, 0.9824580186371794]],
        [60, 0, 0, [-0.6759999999999998, -0.5609999999999998, 0.7430000000000001],
         [-0.6759999999999998, -0.5609999999999998, 0.7430000000000001]],
        [60, 30, 0, [-1.544942286340599, -1.3905855345755218, 0.36300377355803837],
         [-1.1400956521839989, -1.0834897710580573, 0.4335910392920804]],
        [60, 30, 180, [-0.24590418066394135, -0.19893457896813463, 0.8450037735580384],
         [-0.22153699864030738, -0.24086529954064415, 0.7744165078239963]],
    ],
}

# terrain/orientation_test.go:76-101 (TestOrientationCardinal): planes
# z = a*x + b*y + 100 on unit cells; at cell (2, 2) of a 5x5 DEM the
# unweighted and weighted components are exactly these float32 values.
cases["orientation_cardinal"] = {
    "cite": "terrain/orientation_test.go:76-101",
    "rows": [
        {"a": 0, "b": 3, "north": b(1), "east": b(0), "northW": b(3 / math.sqrt(10)), "eastW": b(0)},
        {"a": 0, "b": -3, "north": b(-1), "east": b(0), "northW": b(-3 / math.sqrt(10)), "eastW": b(0)},
        {"a": -2, "b": 0, "north": b(0), "east": b(1), "northW": b(0), "eastW": b(2 / math.sqrt(5))},
    ],
}

if __name__ == "__main__":
    out = os.path.join(HERE, "kat.json")
    with open(out, "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)
    print(out)
