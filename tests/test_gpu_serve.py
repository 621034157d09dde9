"""Serving: requests over a resident mosaic, batched as they arrive, give
each window the result strata_process gives for the window view alone
(bit for bit, data and validity), whatever the mix and the memory budget."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from helpers import assert_same_raster, host_raster, like, to_device, to_host
from strata_b200 import engine, focal, serve, synth, terrain

pytestmark = pytest.mark.gpu

OPS = [
    lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=30)),
    lambda: terrain.aspect_stage(terrain.AspectOptions(CellSize=30)),
    lambda: terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=30)),
    lambda: focal.box_stage(focal.BoxOptions(Radius=5), engine._lib.OP_MEAN),
    lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=terrain.RuggednessTPI)),
]


def _mosaic(w, h, masked=True):
    return host_raster(synth.fbm_dem(w, h, 77), synth.block_mask(w, h, 77, 0.03) if masked else None)


def _requests(rng, W, H, n):
    out = []
    for _ in range(n):
        w = int(np.exp(rng.uniform(np.log(4), np.log(400))))
        h = int(np.exp(rng.uniform(np.log(4), np.log(400))))
        x = int(rng.integers(0, W - w + 1))
        y = int(rng.integers(0, H - h + 1))
        out.append((int(rng.integers(len(OPS))), x, y, w, h))
    return out


def _alone(mosaic_dev, op, x, y, w, h):
    win = mosaic_dev.Window(x, y, w, h)
    dst = to_device(like(to_host(win), masked=mosaic_dev.valid is not None))
    engine.process(OPS[op](), [dst], [win])
    return to_host(dst)


@pytest.mark.parametrize("budget", [0, 4 << 20])
def test_served_equals_alone(budget):
    W, H = 1500, 1300
    m = to_device(_mosaic(W, H))
    srv = serve.Server(m, budget_bytes=budget, streams=3, max_batch=16)
    rng = np.random.default_rng(5)
    reqs = _requests(rng, W, H, 60)
    tickets = []
    # submitted from two threads, so arrivals interleave with running batches
    def submit(part):
        for op, x, y, w, h in part:
            tickets.append((srv.submit(OPS[op](), x, y, w, h), (op, x, y, w, h)))

    th = [threading.Thread(target=submit, args=(reqs[i::2],)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for t, (op, x, y, w, h) in tickets:
        res = srv.wait(t, timeout_ms=60000)
        got = to_host(res.copy())
        assert res.t_submit_ns <= res.t_start_ns <= res.t_done_ns
        srv.release(t)
        want = _alone(m, op, x, y, w, h)
        assert_same_raster(got, want, f"request op={op} at ({x}, {y}) {w}x{h}")
    st = srv.stats()
    assert st["served"] == len(reqs) and st["used_bytes"] == 0
    assert st["batches"] >= 1
    srv.close()


@pytest.mark.parametrize("band", [1, 7, 64])
def test_band_option(band):
    """The server's unit band only changes how radius-1 requests are cut
    into work units: every result equals the window alone at any band, and
    bands outside 0..256 are refused."""
    from strata_b200.raster import StrataPanic

    W, H = 700, 600
    m = to_device(_mosaic(W, H))
    for bad in (-1, 257):
        with pytest.raises(StrataPanic):
            serve.Server(m, band=bad)
    srv = serve.Server(m, band=band, streams=2, max_batch=8)
    reqs = _requests(np.random.default_rng(40 + band), W, H, 20)
    tickets = srv.submit_many([(OPS[o](), x, y, w, h) for o, x, y, w, h in reqs])
    for res, (op, x, y, w, h) in zip(srv.wait_many(tickets, timeout_ms=60000), reqs):
        assert_same_raster(to_host(res.copy()), _alone(m, op, x, y, w, h),
                           f"band={band} op={op} at ({x}, {y}) {w}x{h}")
    srv.release_many(tickets)
    assert srv.stats()["used_bytes"] == 0
    srv.close()


def test_unmasked_mosaic_and_bad_window():
    W, H = 300, 200
    m = to_device(_mosaic(W, H, masked=False))
    srv = serve.Server(m)
    t = srv.submit(OPS[0](), 10, 20, 100, 50)
    got = to_host(srv.wait(t).copy())
    assert_same_raster(got, _alone(m, 0, 10, 20, 100, 50), "unmasked")
    srv.release(t)
    with pytest.raises(engine.StrataPanic, match="outside"):
        srv.submit(OPS[0](), 250, 0, 100, 10)
    srv.close()


def test_submit_many_equals_alone_and_is_all_or_nothing():
    """Requests submitted, waited for and released in groups give each
    window the result strata_process gives it alone; a group with an
    invalid request queues none of its requests."""
    W, H = 900, 700
    m = to_device(_mosaic(W, H))
    srv = serve.Server(m, streams=2, max_batch=8)
    rng = np.random.default_rng(9)
    reqs = _requests(rng, W, H, 30)
    tickets = srv.submit_many([(OPS[op](), x, y, w, h) for op, x, y, w, h in reqs])
    assert len(tickets) == len(reqs) and len(set(tickets)) == len(reqs)
    results = srv.wait_many(tickets, timeout_ms=60000)
    for res, (op, x, y, w, h) in zip(results, reqs):
        assert_same_raster(to_host(res.copy()), _alone(m, op, x, y, w, h), f"group request op={op} at ({x}, {y})")
    srv.release_many(tickets)
    st = srv.stats()
    assert st["served"] == len(reqs) and st["used_bytes"] == 0
    with pytest.raises(engine.StrataPanic, match="outside"):
        srv.submit_many([(OPS[0](), 0, 0, 10, 10), (OPS[1](), W - 5, 0, 10, 10)])
    assert srv.stats()["served"] == len(reqs)
    srv.close()
