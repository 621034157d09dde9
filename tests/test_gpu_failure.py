"""Failure paths on the device, made to happen without a fault: a bounded
device-side wait that runs out reports STRATA_ETIMEDOUT and leaves the
context usable, and a serving wait with no time left reports the request
as not done. Nothing here faults, traps or hangs the GPU: the wait that
runs out is on a barrier nothing arrives at, with a short bound, and the
kernel then waits (bounded) for its own copies before it returns."""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import assert_same_raster, host_raster, like, run_oracle, to_device, to_host
from strata_b200 import _lib, engine, serve, synth, terrain

pytestmark = pytest.mark.gpu


def test_tma_wait_that_runs_out_reports_timeout():
    w, h = 512, 300  # rows 16-byte aligned: the TMA march runs
    src = host_raster(synth.fbm_dem(w, h, 31), synth.block_mask(w, h, 31, 0.02))
    dsrc = to_device(src)
    stages = terrain.slope_stage(terrain.SlopeOptions(CellSize=30))
    dst = to_device(like(src))
    os.environ["STRATA_TEST_STALL_FIRST_WAIT"] = "1"
    try:
        with pytest.raises(RuntimeError, match=f"error {_lib.ETIMEDOUT}"):
            engine.process(stages, [dst], [dsrc])
    finally:
        del os.environ["STRATA_TEST_STALL_FIRST_WAIT"]
    # the status word was read and cleared, and the context still works
    dst = to_device(like(src))
    assert engine.process(stages, [dst], [dsrc]) is None
    want = like(src)
    run_oracle(stages, src, [want])
    assert_same_raster(to_host(dst), want, "after the timeout")


def test_server_wait_with_no_time_left():
    W, H = 3000, 2600
    m = to_device(host_raster(synth.fbm_dem(W, H, 41), synth.block_mask(W, H, 41, 0.02)))
    srv = serve.Server(m, streams=2, max_batch=8)
    stages = terrain.slope_stage(terrain.SlopeOptions(CellSize=30))
    try:
        timed_out = 0
        for i in range(8):
            t = srv.submit(stages, 10 + i, 20, W - 40, H - 60)
            if srv.poll(t) is None:  # strata_server_wait with timeout_ms = 0
                timed_out += 1
            r = srv.wait(t, -1)
            win = m.Window(10 + i, 20, W - 40, H - 60)
            alone = to_device(like(to_host(win)))
            engine.process(stages, [alone], [win])
            assert_same_raster(to_host(r.copy(0)), to_host(alone), f"request {i}")
            srv.release(t)
        assert timed_out > 0
    finally:
        srv.close()
