"""The float32 path's distance from float64 arithmetic, per op (the
oracle's, which the device equals bit for bit): the ops without
cancellation stay within a few float32 ulps, the order-free folds are
exact, and every op's absolute error is small for its value range."""
from __future__ import annotations

import pytest

from oracle import fp64_error


@pytest.fixture(scope="module")
def rows():
    return {r["op"]: r for r in fp64_error.report(256)}


def test_slope_aspect_riley_within_a_few_ulps(rows):
    assert rows["slope (degrees)"]["p99_ulp"] <= 4 and rows["slope (degrees)"]["max_ulp"] <= 8
    assert rows["aspect"]["p99_ulp"] <= 4 and rows["aspect"]["max_abs"] < 1e-4
    assert rows["TRI (Riley)"]["max_ulp"] <= 0.5  # float64 sum, one rounding


def test_order_free_folds_are_exact(rows):
    assert rows["max r3"]["max_abs"] == 0 and rows["max r8"]["max_abs"] == 0
    assert rows["roughness"]["max_ulp"] <= 0.5  # max - min, one rounding


def test_absolute_errors_are_small(rows):
    # values: degrees, 0..255 shades, metres, 1/m curvatures, N(0,1)-scale focal sums
    for op, bound in [("hillshade", 1e-3), ("curvature profile", 1e-4), ("curvature plan", 1e-3),
                      ("curvature mean", 1e-4), ("TPI", 1e-3), ("correlate r3", 1e-4), ("correlate r8", 1e-3),
                      ("mean r3", 1e-5), ("mean r8", 1e-5), ("gaussian r8", 1e-5)]:
        assert rows[op]["max_abs"] < bound, (op, rows[op])
