"""The multi-GPU sharding logic, run as two gloo ranks on the CPU: each rank
computes its row strip (with its halo) as a raster of its own, keeps its
rows, and rank 0 reassembles them; the result equals the whole-raster
result bit for bit, data and validity. The oracle stands in for the device
here (the logic under test is the partition and the halo arithmetic)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _cases():
    from strata_b200 import engine, focal, synth, terrain

    w = synth.uniform_weights(25, 7)
    return [
        ("slope", lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=30)), 1),
        ("mean r3", lambda: focal.box_stage(focal.BoxOptions(Radius=3), engine._lib.OP_MEAN), 3),
        ("correlate r2", lambda: focal.weights_stage(focal.WeightsOptions(2, w), False), 2),
    ]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys

        here = os.path.dirname(os.path.abspath(__file__))
        sys.path.insert(0, here)
        sys.path.insert(0, os.path.dirname(here))
        from helpers import host_raster, like, run_oracle

        from strata_b200 import shard, synth

        W, H = 70, 53
        cells = synth.fbm_dem(W, H, 11)
        valid = synth.cell_mask(W, H, 11, 0.02)
        results = {}
        for name, mk, r in _cases():
            y0, y1 = shard.strips(H, world)[rank]
            s0, s1 = shard.halo_rows(H, r, y0, y1)
            src = host_raster(np.ascontiguousarray(cells[s0:s1]), valid[s0:s1])
            dst = like(src)
            run_oracle(mk(), src, [dst])
            k0, k1 = shard.kept_rows(H, r, y0, y1)
            mine = (dst.numpy()[k0:k1], dst.valid_numpy()[k0:k1])
            gathered = [None] * world
            dist.all_gather_object(gathered, mine)
            if rank == 0:
                results[name] = (np.concatenate([g[0] for g in gathered]),
                                 np.concatenate([g[1] for g in gathered]))
        t = shard.max_over_ranks(float(rank + 1))
        if rank == 0:
            out.put(("ok", results, t))
    except Exception as e:  # report to the parent
        out.put(("error", repr(e), None))
        raise
    finally:
        dist.destroy_process_group()


def test_two_rank_strips_equal_whole_raster():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from helpers import host_raster, like, run_oracle, same_bits

    from strata_b200 import synth

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    status, results, tmax = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
    assert status == "ok", results
    assert tmax == 2.0
    W, H = 70, 53
    src = host_raster(synth.fbm_dem(W, H, 11), synth.cell_mask(W, H, 11, 0.02))
    for name, mk, r in _cases():
        want = like(src)
        run_oracle(mk(), src, [want])
        data, val = results[name]
        assert same_bits(data, want.numpy()).all(), name
        assert (val == want.valid_numpy()).all(), name


def test_strip_arithmetic():
    from strata_b200 import shard

    assert shard.strips(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert shard.halo_rows(10, 2, 4, 7) == (2, 9)
    assert shard.kept_rows(10, 2, 4, 7) == (2, 5)
    assert shard.halo_rows(10, 2, 0, 4) == (0, 6) and shard.kept_rows(10, 2, 0, 4) == (0, 4)
    a = shard.assign_rasters([5, 100, 7, 60, 50], 2)
    assert sorted(a[0] + a[1]) == [0, 1, 2, 3, 4]
    loads = [sum([5, 100, 7, 60, 50][i] for i in r) for r in a]
    assert max(loads) - min(loads) <= 100


def _oracle_strip(stages, dsts, src, height, src_row, dst_row, opts=None):
    """Stands in for engine.process_strip on a rank without a GPU: the
    oracle over the strip's source rows as a raster of its own, its rows
    dst_row.. kept (the strip's own edge rows are the halo or the whole
    raster's edge)."""
    from helpers import like, run_oracle

    from strata_b200 import engine

    full = [like(src) for _ in dsts]
    run_oracle(stages, src, full)
    k0 = dst_row - src_row
    for d, f in zip(dsts, full):
        engine._copy_cells(d, f.Window(0, k0, f.width, d.height), d.valid is not None)


def _rank_product(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys

        here = os.path.dirname(os.path.abspath(__file__))
        sys.path.insert(0, here)
        sys.path.insert(0, os.path.dirname(here))
        from helpers import host_raster, like

        from strata_b200 import shard, synth

        W, H = 70, 53
        src = host_raster(synth.fbm_dem(W, H, 11), synth.cell_mask(W, H, 11, 0.02), W + 3, 9)
        results = {}
        for name, mk, r in _cases():
            dst = like(src, W + 1, 17)
            shard.process_sharded(mk(), [dst], src, rank, world, compute=_oracle_strip)
            results[name] = (dst.numpy(), dst.valid_numpy(), shard.stage_radius(mk()))
        out.put((rank, "ok", results))
    except Exception as e:  # report to the parent
        out.put((rank, "error", repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def test_two_rank_product_sharding_equals_whole_raster():
    """shard.process_sharded, the product's multi-process split, over two
    gloo ranks: each rank computes its strip (the oracle standing in for
    its GPU) and after the exchange both ranks hold the whole result, equal
    to the whole-raster oracle bit for bit."""
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from helpers import host_raster, like, run_oracle, same_bits

    from strata_b200 import synth

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_product, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    W, H = 70, 53
    src = host_raster(synth.fbm_dem(W, H, 11), synth.cell_mask(W, H, 11, 0.02), W + 3, 9)
    for rank, status, results in got:
        assert status == "ok", results
        for name, mk, r in _cases():
            want = like(src)
            run_oracle(mk(), src, [want])
            data, val, radius = results[name]
            assert radius == r, name
            assert same_bits(data, want.numpy()).all(), (rank, name)
            assert (val == want.valid_numpy()).all(), (rank, name)
