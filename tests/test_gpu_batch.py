"""Batches: every raster's result in a batch of mixed sizes, ops, masks
and tile shapes equals its result alone (strata_process) and the oracle's,
bit for bit; the autotuner picks one of its candidate shapes."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import assert_same_raster, host_raster, like, run_oracle, to_device, to_host
from strata_b200 import batch, engine, focal, synth, terrain, transfer

pytestmark = pytest.mark.gpu


def _ops(rng):
    r = int(rng.integers(1, 9))
    w = synth.uniform_weights((2 * r + 1) ** 2, int(rng.integers(1 << 30)))
    choices = [
        (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=float(rng.uniform(1, 90)))), 1),
        (lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=float(rng.uniform(1, 90)))), 1),
        (lambda: terrain.curvature_stage(terrain.CurvatureOptions(CellSize=float(rng.uniform(1, 90)),
                                                                  Type=int(rng.integers(3)))), 1),
        (lambda: focal.weights_stage(focal.WeightsOptions(r, w), False), 1),
        (lambda: focal.box_stage(focal.BoxOptions(int(rng.integers(1, 9))), engine._lib.OP_MEAN), 1),
        (lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=int(rng.integers(4)),
                                                                    Radius=int(rng.integers(1, 9)))), 1),
        (lambda: focal.separable_stage(focal.SeparableOptions(3, focal.Gaussian(3, 1.5), synth.uniform_weights(7, 5))),
         1),
        (lambda: terrain.gradient_stage(terrain.GradientOptions(CellSize=30)), 2),
        (lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=10)).extend(
            transfer.lookup_stage([0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5])).extend(
            transfer.reclass_stage([1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5])), 1),
    ]
    make, nout = choices[int(rng.integers(len(choices)))]
    return make(), nout


def test_batch_equals_alone_and_oracle():
    rng = np.random.default_rng(42)
    items, want, srcs = [], [], []
    shapes = [(64, 32), (128, 16), (32, 64), (100, 7), None]
    for i in range(40):
        w = int(np.exp(rng.uniform(np.log(3), np.log(300))))
        h = int(np.exp(rng.uniform(np.log(3), np.log(300))))
        masked = bool(rng.integers(2))
        src = host_raster(synth.fbm_dem(w, h, 100 + i), synth.cell_mask(w, h, i, 0.02) if masked else None)
        stages, nout = _ops(rng)
        outs = [like(src) for _ in range(nout)]
        run_oracle(stages, src, outs)
        dsrc = to_device(src)
        douts = [to_device(like(src)) for _ in range(nout)]
        items.append(batch.Item(stages, dsrc, douts, shapes[i % len(shapes)]))
        want.append(outs)
        srcs.append((dsrc, stages, nout, src))
    b = batch.Batch(items)
    b.run()
    st, classes = b.stats()
    assert classes >= 5 and st.Cells == sum(it.src.width * it.src.height for it in items)
    for i, it in enumerate(items):
        for k, d in enumerate(it.dst):
            assert_same_raster(to_host(d), want[i][k], f"batch raster {i} out {k}")
    # the same rasters alone, through strata_process
    for i, (dsrc, stages, nout, src) in enumerate(srcs):
        alone = [to_device(like(src)) for _ in range(nout)]
        engine.process(stages, alone, [dsrc])
        for k in range(nout):
            assert_same_raster(to_host(alone[k]), want[i][k], f"alone raster {i}")
    # run again: the graph replays with the same bits
    for it in items:
        for d in it.dst:
            d.data.fill_(7.0)
    b.run()
    for i, it in enumerate(items):
        for k, d in enumerate(it.dst):
            assert_same_raster(to_host(d), want[i][k], f"replay raster {i}")
    b.close()


def test_autotuner_picks_a_candidate(tmp_path):
    import torch

    tuner = batch.Autotuner(path=str(tmp_path / "tune.json"), probe=512, reps=2)
    st = terrain.slope_stage(terrain.SlopeOptions(CellSize=30))
    tuner.register(st)
    shape = tuner.shape(batch._class_key(st))
    assert tuple(shape) in batch.CANDIDATES
    assert (tmp_path / "tune.json").exists()
    n = 300
    src = to_device(host_raster(synth.fbm_dem(n, n, 3)))
    dst = to_device(like(to_host(src)))
    b = batch.Batch([batch.Item(st, src, [dst])], tuner=tuner)
    b.run()
    want = like(to_host(src))
    run_oracle(st, to_host(src), [want])
    assert_same_raster(to_host(dst), want, "tuned")
    torch.cuda.synchronize()


def test_batch_rejects_host_rasters():
    src = host_raster(synth.fbm_dem(16, 16, 1))
    with pytest.raises(engine.StrataPanic, match="must be on the device"):
        batch.Batch([batch.Item(terrain.slope_stage(terrain.SlopeOptions(CellSize=1)), src, [like(src)])])
