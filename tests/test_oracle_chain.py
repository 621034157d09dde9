"""The oracle's vec.Chain (internal/vec/chain.go, scalar.go) against numpy's
float32 arithmetic, op by op, and its pointwise validity rule (the AND of
the masked inputs, halo.go:213-229 at reach 0). No GPU."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as orc

SPECIALS = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-45, -1e-45, 1.17549435e-38, 3.4028235e38, 1.0, -1.0,
                     0.5, 2.0, -7.25, 1e30, -3e-39], np.float32)


def _r(a, valid=None, off=0):
    h, w = a.shape
    return dict(data=np.ascontiguousarray(a), width=w, height=h, stride=w,
                valid=valid, valid_offset=off)


def run(steps, *inputs, masks=None):
    h, w = inputs[0].shape
    out = np.zeros((h, w), np.float32)
    srcs = [_r(a, None if masks is None else masks[i]) for i, a in enumerate(inputs)]
    dmask = None if masks is None else np.zeros((h * w + 63) // 64 + 1, np.uint64)
    orc.process_n([orc.step_stage(*s) for s in steps], srcs, [_r(out, dmask)])
    return out, dmask


def same(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())


def go_min(a, b):
    """Go's min: NaN wins, -0 below +0."""
    r = np.where(a < b, a, b)
    r = np.where((a == 0) & (b == 0), np.where(np.signbit(a), a, b), r)
    return np.where(np.isnan(a) | np.isnan(b), np.float32(np.nan), r).astype(np.float32)


def go_max(a, b):
    r = np.where(a > b, a, b)
    r = np.where((a == 0) & (b == 0), np.where(np.signbit(a), b, a), r)
    return np.where(np.isnan(a) | np.isnan(b), np.float32(np.nan), r).astype(np.float32)


def pairs():
    a, b = np.meshgrid(SPECIALS, SPECIALS)
    return a.astype(np.float32), b.astype(np.float32)


def test_binary_ops():
    a, b = pairs()
    with np.errstate(all="ignore"):
        assert same(run([(orc.VEC_ADD, 1)], a, b)[0], a + b)
        assert same(run([(orc.VEC_SUB, 1)], a, b)[0], a - b)
        assert same(run([(orc.VEC_MUL, 1)], a, b)[0], a * b)
        assert same(run([(orc.VEC_DIV, 1)], a, b)[0], a / b)
    assert same(run([(orc.VEC_MIN, 1)], a, b)[0], go_min(a, b))
    assert same(run([(orc.VEC_MAX, 1)], a, b)[0], go_max(a, b))
    # the sign of zero, bit for bit
    z = np.array([[0.0, -0.0]], np.float32)
    nz = np.array([[-0.0, 0.0]], np.float32)
    assert (run([(orc.VEC_MIN, 1)], z, nz)[0].view(np.uint32) == np.uint32(0x80000000)).all()
    assert (run([(orc.VEC_MAX, 1)], z, nz)[0].view(np.uint32) == 0).all()


def test_unary_ops():
    a = SPECIALS.reshape(1, -1)
    with np.errstate(all="ignore"):
        assert same(run([(orc.VEC_ADD_SCALAR, -1, 2.5)], a)[0], a + np.float32(2.5))
        assert same(run([(orc.VEC_MUL_SCALAR, -1, -3.0)], a)[0], a * np.float32(-3.0))
        assert same(run([(orc.VEC_AFFINE, -1, 1.1, -0.3)], a)[0], (a * np.float32(1.1)) + np.float32(-0.3))
        assert same(run([(orc.VEC_SUB_DIV, -1, -1.5, 7.0)], a)[0], (a - np.float32(-1.5)) / np.float32(7.0))
        assert same(run([(orc.VEC_SQRT, -1)], a)[0], np.sqrt(a.astype(np.float64)).astype(np.float32))
    assert same(run([(orc.VEC_CLAMP, -1, -10.0, 10.0)], a)[0],
                go_min(go_max(a, np.float32(-10)), np.float32(10)))
    got = run([(orc.VEC_ABS, -1)], a)[0]
    assert (got.view(np.uint32) == (a.view(np.uint32) & np.uint32(0x7FFFFFFF))).all()  # NaN payloads kept


def test_affine_is_two_roundings():
    """Affine is float32(v*a) + b, not a fused multiply-add: pick cells where
    the two differ and check the unfused result."""
    rng = np.random.default_rng(3)
    v = rng.standard_normal(4096).astype(np.float32).reshape(64, 64)
    a, b = np.float32(1.0 + 2 ** -12), np.float32(-1.0)
    unfused = (v * a) + b
    fused = (v.astype(np.float64) * np.float64(a) + np.float64(b)).astype(np.float32)
    assert not same(unfused, fused)  # the inputs tell the two apart
    assert same(run([(orc.VEC_AFFINE, -1, float(a), float(b))], v)[0], unfused)


def test_subdiv_endpoints_exact():
    """SubDiv subtracts before it divides (internal/vec/scalar.go:74-83):
    lo gives exactly 0 and lo + span exactly 1."""
    lo, span = np.float32(0.1), np.float32(0.7)
    v = np.array([[lo, lo + span]], np.float32)
    out = run([(orc.VEC_SUB_DIV, -1, float(lo), float(span))], v)[0]
    assert out[0, 0] == 0 and out[0, 1] == np.float32((lo + span - lo) / span)


def test_chain_order_and_validity():
    rng = np.random.default_rng(5)
    h, w = 9, 70
    x = [rng.standard_normal((h, w)).astype(np.float32) for _ in range(3)]
    m = [orc.pack_mask(rng.random((h, w)) > 0.2), None, orc.pack_mask(rng.random((h, w)) > 0.3)]
    steps = [(orc.VEC_ADD, 1), (orc.VEC_MUL_SCALAR, -1, 0.5), (orc.VEC_MAX, 2), (orc.VEC_SQRT, -1)]
    out, dmask = run(steps, *x, masks=m)
    with np.errstate(invalid="ignore"):
        want = np.sqrt(go_max((x[0] + x[1]) * np.float32(0.5), x[2]).astype(np.float64)).astype(np.float32)
    assert same(out, want)
    bits = lambda mm: np.unpackbits(mm.view(np.uint8), bitorder="little")[:h * w].astype(bool)
    assert (bits(dmask) == (bits(m[0]) & bits(m[2]))).all()


def test_oracle_rejects_what_new_chain_panics_on():
    a = np.zeros((2, 3), np.float32)
    with pytest.raises(ValueError):
        run([(orc.VEC_ADD, 2)], a, a)  # input 2 of 2
    with pytest.raises(ValueError):
        run([(orc.VEC_ABS, 0)], a)  # a unary step names an input
    with pytest.raises(ValueError):
        run([(13, -1)], a)  # unknown op
    out = np.zeros((2, 3), np.float32)
    with pytest.raises(ValueError):  # a stencil-led pipeline takes one input
        orc.process_n([orc.slope_stage(), orc.step_stage(orc.VEC_ABS)], [_r(a), _r(a)], [_r(out)])
