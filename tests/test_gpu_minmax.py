"""Pins the device's Go min / max (NaN wins, -0 orders below +0) on every
ordered pair of special values, through focal Min / Max at radius 1 and
roughness, against the oracle's restatement of Go's rules (the pairs of
the reference's TestSIMDMinMaxEdgePairs, internal/focalrow/simd_test.go)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import assert_same_raster, host_raster, like, run_oracle, to_device, to_host
from strata_b200 import engine, focal, terrain

pytestmark = pytest.mark.gpu

SPECIALS = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 3.4e38, -3.4e38, 2.5],
                    np.float32)


def pair_raster():
    """3 rows, one 3x3 block per ordered pair (a, b): eight a's around a
    centre b, so each block's min / max is Go's min(a, b) / max(a, b)."""
    n = len(SPECIALS)
    cells = np.zeros((3, 3 * n * n + 4), np.float32)  # width a multiple of 4: the marching kernel
    for i, a in enumerate(SPECIALS):
        for j, b in enumerate(SPECIALS):
            c = 3 * (i * n + j)
            cells[:, c:c + 3] = a
            cells[1, c + 1] = b
    return cells


@pytest.mark.parametrize("device", [False, True])
def test_min_max_special_pairs(device):
    src = host_raster(pair_raster())
    for stages in (focal.box_stage(focal.BoxOptions(Radius=1), engine._lib.OP_MIN),
                   focal.box_stage(focal.BoxOptions(Radius=1), engine._lib.OP_MAX),
                   terrain.ruggedness_stage(terrain.RuggednessOptions(Type=terrain.RuggednessRoughness))):
        want = like(src)
        run_oracle(stages, src, [want])
        got = like(src)
        if device:
            d = to_device(got)
            engine.process(stages, [d], [to_device(src)])
            got = to_host(d)
        else:
            engine.process(stages, [got], [src])
        assert_same_raster(got, want, "special pairs")
