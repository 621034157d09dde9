"""vec.Chain on the device (internal/vec/chain.go, internal/exec/pipeline.go:
432-490): every step op alone and in long chains over up to four inputs,
the unary steps fused after a stencil, the algebra and transfer.Rescale
entry points, and the batched and chunked forms, each against the oracle
cell for cell and bit for bit in the masks (rastertest.SameFloat)."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from helpers import (assert_padding_untouched, assert_same_raster, host_raster, like, poison, run_oracle, to_device,
                     to_host)
from strata_b200 import algebra, engine, focal, graph, synth, terrain, transfer, vec
from strata_b200.raster import Float32Raster, NotSupported, StrataPanic

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (3, 3), (17, 5), (61, 37), (300, 9), (1028, 33)]
SPECIALS = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-45, -1e-45, 1.17549435e-38, 3.4028235e38, -3.4028235e38,
                     1.0, -1.0, 0.5, 2.0, -7.25], np.float32)


def cells_for(w, h, seed):
    """Normal values with specials planted: NaN, +-Inf, +-0, subnormals and
    the float32 extremes."""
    rng = np.random.default_rng(seed)
    c = (rng.standard_normal((h, w)) * 50).astype(np.float32)
    pick = rng.random((h, w)) < 0.2
    c[pick] = SPECIALS[rng.integers(0, SPECIALS.size, int(pick.sum()))]
    return c


def input_layouts(w, h, n, seed, masked):
    """n inputs with their own strides, bit offsets and masks."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        stride = w + int(rng.integers(0, 9)) * (i % 2)
        offset = int(rng.integers(0, 64)) if i % 2 else 0
        valid = synth.cell_mask(w, h, seed + 7 * i, 0.05) if masked and (i != 1 or n == 2) else None
        out.append(host_raster(cells_for(w, h, seed + 100 * i), valid, stride, offset))
    return out


def check_chain(stages, srcs, dst_stride=None, dst_offset=0, masked=None, device=False, what=""):
    want = like(srcs[0], dst_stride, dst_offset, masked=masked if masked is not None else
                any(s.valid is not None for s in srcs))
    got = like(srcs[0], dst_stride, dst_offset, masked=want.valid is not None)
    before = Float32Raster(np.array(got.data), got.width, got.height, got.stride,
                           None if got.valid is None else np.array(got.valid), got.valid_offset)
    run_oracle(stages, list(srcs), [want])
    if device:
        dgot = to_device(got)
        assert engine.process(stages, [dgot], [to_device(s) for s in srcs]) is None
        got = to_host(dgot)
    else:
        assert engine.process(stages, [got], list(srcs)) is None
    assert_same_raster(got, want, what)
    assert_padding_untouched(before, got, what)


UNARY = [(vec.OpAddScalar, 2.5, 0), (vec.OpMulScalar, -3.0, 0), (vec.OpAffine, 1.1, -0.3),
         (vec.OpAffine, 0.0, -0.0), (vec.OpSubDiv, -1.5, 7.0), (vec.OpSubDiv, 0.0, 0.0), (vec.OpClamp, -10.0, 10.0),
         (vec.OpClamp, 3.0, -3.0), (vec.OpAbs, 0, 0), (vec.OpSqrt, 0, 0)]
BINARY = [vec.OpAdd, vec.OpSub, vec.OpMul, vec.OpDiv, vec.OpMin, vec.OpMax]


@pytest.mark.parametrize("op,k0,k1", UNARY)
def test_unary_step(op, k0, k1):
    for (w, h), masked, device in itertools.product(SHAPES, (False, True), (False, True)):
        srcs = input_layouts(w, h, 1, w * 3 + h, masked)
        check_chain(vec.step_stage(op, -1, k0, k1), srcs, w + 3, 21, device=device,
                    what=f"{vec.op_name(op)} {w}x{h} masked={masked} device={device}")


@pytest.mark.parametrize("op", BINARY)
def test_binary_step(op):
    for (w, h), masked, device in itertools.product(SHAPES, (False, True), (False, True)):
        srcs = input_layouts(w, h, 2, w + 5 * h, masked)
        check_chain(vec.step_stage(op, 1), srcs, None, 45, device=device,
                    what=f"{vec.op_name(op)} {w}x{h} masked={masked} device={device}")


def test_binary_step_reads_its_own_start():
    """A binary step may name input 0, the chain's own start (v op v)."""
    srcs = input_layouts(257, 31, 1, 4, True)
    for op in BINARY:
        check_chain(vec.step_stage(op, 0), srcs, what=vec.op_name(op))


def test_long_chain_over_four_inputs():
    """vec.MaxSteps steps over four inputs, with a Lookup and a Reclass in
    the middle of the sequence (one pass, the running value carried)."""
    rng = np.random.default_rng(9)
    for (w, h), masked in itertools.product([(3, 3), (129, 67), (1028, 33)], (False, True)):
        srcs = input_layouts(w, h, 4, w + h, masked)
        st = engine.StageList()
        ops = [vec.step_stage(vec.OpAdd, 1), vec.step_stage(vec.OpMulScalar, -1, 0.5),
               vec.step_stage(vec.OpMax, 2), transfer.lookup_stage([-50, 0, 10, 80], [1, 0, 2, -3]),
               vec.step_stage(vec.OpSub, 3), vec.step_stage(vec.OpAbs), vec.step_stage(vec.OpSqrt),
               vec.step_stage(vec.OpAffine, -1, 3.0, -1.0), vec.step_stage(vec.OpMin, 1),
               transfer.reclass_stage([-1, 0.5, 2], [10, 20, 30, 40]), vec.step_stage(vec.OpDiv, 2),
               vec.step_stage(vec.OpSubDiv, -1, 0.25, 3.0), vec.step_stage(vec.OpClamp, -1, -5, 5),
               vec.step_stage(vec.OpMul, 0), vec.step_stage(vec.OpAddScalar, -1, float(rng.standard_normal())),
               vec.step_stage(vec.OpAdd, 3)]
        for o in ops:
            st.extend(o)
        assert len(st.stages) == vec.MaxSteps
        check_chain(st, srcs, what=f"chain16 {w}x{h} masked={masked}")
        check_chain(st, srcs, device=True, what=f"chain16 {w}x{h} masked={masked} device")


def test_chain_with_unread_inputs_and_masked_output_of_unmasked_inputs():
    """Inputs the steps never name are still checked and still count in the
    validity; unmasked inputs into a masked output give all-valid cells."""
    w, h = 200, 17
    srcs = input_layouts(w, h, 3, 1, True)
    check_chain(vec.step_stage(vec.OpAdd, 1), srcs, what="unread input 2")
    plain = [host_raster(cells_for(w, h, 3 + i)) for i in range(2)]
    check_chain(vec.step_stage(vec.OpSub, 1), plain, w + 7, 63, masked=True, what="masked out, unmasked in")


def test_new_chain_from_another_first():
    w, h = 131, 29
    srcs = input_layouts(w, h, 3, 5, True)
    steps = [vec.Step(vec.OpSub, 0), vec.Step(vec.OpMul, 2), vec.Step(vec.OpAbs)]
    ch = vec.NewChain(3, 1, steps)
    got = like(srcs[0], masked=True)
    assert ch.Run(got, srcs) is None
    # the same chain written from input 0, by hand: acc = srcs[1]
    want = like(srcs[0], masked=True)
    run_oracle(_by_hand(), [srcs[1], srcs[0], srcs[2]], [want])
    assert_same_raster(got, want, "NewChain first=1")


def _by_hand():
    st = engine.StageList()
    for o in (vec.step_stage(vec.OpSub, 1), vec.step_stage(vec.OpMul, 2), vec.step_stage(vec.OpAbs)):
        st.extend(o)
    return st


def test_new_chain_checks():
    with pytest.raises(StrataPanic, match="needs at least one"):
        vec.NewChain(0, 0, [vec.Step(vec.OpAbs)])
    with pytest.raises(StrataPanic, match="not one of its 2"):
        vec.NewChain(2, 2, [vec.Step(vec.OpAbs)])
    with pytest.raises(StrataPanic, match="no steps"):
        vec.NewChain(1, 0, [])
    with pytest.raises(StrataPanic, match="at most 16"):
        vec.NewChain(1, 0, [vec.Step(vec.OpAbs)] * 17)
    with pytest.raises(StrataPanic, match="reads input 3"):
        vec.NewChain(2, 0, [vec.Step(vec.OpAdd, 3)])
    with pytest.raises(StrataPanic, match="Src must be -1"):
        vec.NewChain(2, 0, [vec.Step(vec.OpSqrt, 1)])
    src = host_raster(cells_for(10, 4, 1))
    with pytest.raises(StrataPanic, match="takes 2 inputs"):
        vec.NewChain(2, 0, [vec.Step(vec.OpAdd, 1)]).Run(like(src), [src])
    # a binary step names an input the call does not pass
    with pytest.raises(StrataPanic, match="kernel takes 2 inputs"):
        engine.process(vec.step_stage(vec.OpAdd, 1), [like(src)], [src])


# ---------------------------------------------------------------------------
# Unary steps fused after a stencil: the staged pipeline's bits (a chain
# step is the kernel its stage runs alone, internal/exec/kernel.go:72-90).

def dem_cells(w, h, seed):
    return poison(synth.fbm_dem(w, h, seed, lo=0, hi=3000), seed, 0.003)


def _tail(*parts):
    st = engine.StageList()
    for p in parts:
        st.extend(p)
    return st


FUSED = {
    "slope_rescale_clamp_reclass": lambda: _tail(terrain.slope_stage(terrain.SlopeOptions(CellSize=30)),
                                                 transfer.rescale_stage(0.1, -0.5), algebra.clamp_stage(0, 3),
                                                 transfer.reclass_stage([0.5, 1, 2], [1, 2, 3, 4])),
    "slope_percent_sqrt": lambda: _tail(terrain.slope_stage(terrain.SlopeOptions(CellSize=10,
                                                                                 Units=terrain.SlopePercent)),
                                        vec.step_stage(vec.OpSqrt)),
    "aspect_subdiv": lambda: _tail(terrain.aspect_stage(terrain.AspectOptions(CellSize=10)),
                                   vec.step_stage(vec.OpSubDiv, -1, 0.0, 360.0)),
    "hillshade_rescale_range": lambda: _tail(terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10)),
                                             transfer.rescale_range_stage(0, 255, -1, 1)),
    "curvature_abs_sqrt": lambda: _tail(terrain.curvature_stage(terrain.CurvatureOptions(CellSize=10, Type=2)),
                                        vec.step_stage(vec.OpAbs), vec.step_stage(vec.OpSqrt)),
    "gradient_only_first_rejected": None,
    "tpi_lookup_affine": lambda: _tail(terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2)),
                                       transfer.lookup_stage([-5, 0, 5], [0, 1, 4]),
                                       vec.step_stage(vec.OpAffine, -1, 2.0, 1.0)),
    "mean_r5_addscalar": lambda: _tail(focal.box_stage(focal.BoxOptions(Radius=5), engine._lib.OP_MEAN),
                                       vec.step_stage(vec.OpAddScalar, -1, -0.25)),
    "gaussian_r8_clamp": lambda: _tail(focal.separable_stage(focal.SeparableOptions(
        Radius=8, Row=focal.Gaussian(8, 2.5), Col=focal.Gaussian(8, 2.5))), algebra.clamp_stage(-1, 1)),
    "fit_slope_rescale": lambda: _tail(terrain.slope_stage(terrain.SlopeOptions(CellSize=10, FitRadius=3)),
                                       transfer.rescale_stage(2.0, 0.0)),
}


@pytest.mark.parametrize("name", sorted(k for k, v in FUSED.items() if v))
def test_stencil_then_unary_steps(name):
    from test_gpu_parity import layouts

    for (w, h), masked, device in itertools.product([(3, 3), (61, 37), (257, 131), (1028, 33)], (False, True),
                                                    (False, True)):
        cells = dem_cells(w, h, w + h)
        for li, lay in enumerate(layouts(w, h, w * h, masked)):
            src = host_raster(cells, lay["src"]["valid"], lay["src"]["stride"], lay["src"]["offset"])
            want = like(src, lay["dst"]["stride"], lay["dst"]["offset"], masked=lay["dst"]["masked"])
            got = like(src, lay["dst"]["stride"], lay["dst"]["offset"], masked=lay["dst"]["masked"])
            run_oracle(FUSED[name](), src, [want])
            if device:
                dg = to_device(got)
                assert engine.process(FUSED[name](), [dg], [to_device(src)]) is None
                got = to_host(dg)
            else:
                assert engine.process(FUSED[name](), [got], [src]) is None
            assert_same_raster(got, want, f"{name} {w}x{h} masked={masked} device={device} layout={li}")


def test_stencil_tail_equals_staged_calls():
    """The fused tail writes what the stages write run one at a time."""
    w, h = 513, 77
    src = host_raster(dem_cells(w, h, 3), synth.block_mask(w, h, 3, 0.05))
    fused = like(src)
    engine.process(FUSED["slope_rescale_clamp_reclass"](), [fused], [src])
    a, b, c = like(src), like(src), like(src)
    terrain.Slope(a, src, terrain.SlopeOptions(CellSize=30))
    transfer.Rescale(b, a, 0.1, -0.5)
    algebra.Clamp(c, b, 0, 3)
    d = like(src)
    transfer.Reclass(d, c, [0.5, 1, 2], [1, 2, 3, 4])
    assert_same_raster(fused, d, "fused vs staged")


def test_binary_step_after_a_stencil_is_not_supported():
    src = host_raster(dem_cells(20, 10, 1))
    st = _tail(terrain.slope_stage(terrain.SlopeOptions(CellSize=1)), vec.step_stage(vec.OpMul, 1))
    with pytest.raises(NotSupported, match="second input"):
        engine.process(st, [like(src)], [src, src])


def test_graph_lowers_rescale_and_clamp_into_the_pass():
    w, h = 300, 40
    src = host_raster(dem_cells(w, h, 8), synth.block_mask(w, h, 8, 0.03))
    g = graph.New()
    dem = g.Input("dem")
    out = graph.Clamp(graph.RescaleRange(graph.Hillshade(dem, terrain.HillshadeOptions(CellSize=10)), 0, 255, 0, 1),
                      0.2, 0.8)
    g.Output("shade", out)
    got = like(src)
    g.Plan().Run(engine.Background(), {"dem": src}, {"shade": got}, engine.Options())
    want = like(src)
    run_oracle(_tail(terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10)),
                     transfer.rescale_range_stage(0, 255, 0, 1), algebra.clamp_stage(0.2, 0.8)), src, [want])
    assert_same_raster(got, want, "graph")


# ---------------------------------------------------------------------------
# The algebra and transfer entry points.

def test_algebra_and_rescale_entry_points():
    w, h = 129, 67
    a, b = input_layouts(w, h, 2, 11, True)
    cases = [(algebra.Add, vec.OpAdd), (algebra.Sub, vec.OpSub), (algebra.Mul, vec.OpMul),
             (algebra.Min, vec.OpMin), (algebra.Max, vec.OpMax)]
    for fn, op in cases:
        got, want = like(a), like(a)
        fn(got, a, b)
        run_oracle(vec.step_stage(op, 1), [a, b], [want])
        assert_same_raster(got, want, fn.__name__)
    got, want = like(a), like(a)
    algebra.Clamp(got, a, -3, 4)
    run_oracle(vec.step_stage(vec.OpClamp, -1, -3, 4), [a], [want])
    assert_same_raster(got, want, "Clamp")
    got, want = like(a), like(a)
    transfer.Rescale(got, a, 0.75, 2.0)
    run_oracle(vec.step_stage(vec.OpAffine, -1, 0.75, 2.0), [a], [want])
    assert_same_raster(got, want, "Rescale")
    from oracle import oracle as orc

    ka, kb = orc.rescale_range_coeffs(-3, 7, 10, 0)
    got, want = like(a), like(a)
    transfer.RescaleRange(got, a, -3, 7, 10, 0)
    run_oracle(vec.step_stage(vec.OpAffine, -1, float(ka), float(kb)), [a], [want])
    assert_same_raster(got, want, "RescaleRange")


def test_mask_copies_values_and_ands_validity():
    """algebra.Mask (algebra/algebra.go:33-46): src's cells, valid where src
    and mask are both valid; mask's values are never read."""
    w, h = 97, 23
    src = host_raster(cells_for(w, h, 1), synth.cell_mask(w, h, 1, 0.1))
    mask = host_raster(np.full((h, w), np.nan, np.float32), synth.cell_mask(w, h, 2, 0.3), w + 3, 17)
    got = like(src)
    algebra.Mask(got, src, mask)
    assert same_or_nan(got.numpy(), src.numpy())
    want_valid = src.valid_numpy() & mask.valid_numpy()
    assert (got.valid_numpy() == want_valid).all()


def same_or_nan(a, b):
    return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())


# ---------------------------------------------------------------------------
# Batched and chunked forms with a unary tail.

def test_chunked_unary_chain_equals_plain():
    w, h = 700, 300
    src = host_raster(dem_cells(w, h, 4), synth.block_mask(w, h, 4, 0.02))
    st = lambda: _tail(terrain.slope_stage(terrain.SlopeOptions(CellSize=30)), transfer.rescale_stage(0.5, 1),
                       algebra.clamp_stage(1, 20))
    plain, chunked = like(src), like(src)
    engine.process(st(), [plain], [src])
    engine.process_chunked(st(), [engine.MemorySink(chunked)], [engine.MemorySource(src)],
                           engine.Options(TileWidth=256, TileHeight=128))
    assert_same_raster(chunked, plain, "chunked")
    pw, cw = like(src), like(src)
    engine.process(_tail(vec.step_stage(vec.OpAbs), vec.step_stage(vec.OpSqrt)), [pw], [src])
    engine.process_chunked(_tail(vec.step_stage(vec.OpAbs), vec.step_stage(vec.OpSqrt)), [engine.MemorySink(cw)],
                           [engine.MemorySource(src)], engine.Options(TileWidth=300, TileHeight=100))
    assert_same_raster(cw, pw, "chunked pointwise")


def test_batch_unary_chain_equals_plain():
    from strata_b200 import batch

    rng = np.random.default_rng(12)
    items, outs, wants = [], [], []
    for i in range(6):
        w, h = int(rng.integers(40, 700)), int(rng.integers(20, 300))
        src = to_device(host_raster(dem_cells(w, h, i), synth.block_mask(w, h, i, 0.02)))
        st = _tail(terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=10)),
                   transfer.rescale_range_stage(0, 255, 0, 1), algebra.clamp_stage(0.1, 0.9))
        out = to_device(like(to_host(src)))
        want = like(to_host(src))
        engine.process(st, [want], [to_host(src)])
        items.append(batch.Item(st, src, [out]))
        outs.append(out)
        wants.append(want)
    b = batch.Batch(items)
    b.run()
    b.close()
    for i, (o, w_) in enumerate(zip(outs, wants)):
        assert_same_raster(to_host(o), w_, f"batch item {i}")
