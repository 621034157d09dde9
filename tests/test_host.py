"""Host-side logic without a GPU: graph lowering, options, Stats and the
raster model's checks."""
from __future__ import annotations

import numpy as np
import pytest

from strata_b200 import engine, focal, graph, terrain
from strata_b200.raster import (Float32Raster, NewFloat32, NewFloat32Like, NotSupported, StrataPanic,
                                mask_from_bool)

XS, YS = [0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5]
BREAKS, VALUES = [1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5]


def test_graph_lowers_slope_lookup_reclass_to_one_pass():
    g = graph.New()
    dem = g.Input("dem")
    cls = graph.Reclass(graph.Lookup(graph.Slope(dem, terrain.SlopeOptions(CellSize=10)), XS, YS), BREAKS, VALUES)
    g.Output("class", cls)
    g.Output("slope", graph.Slope(dem, terrain.SlopeOptions(CellSize=10)))
    p = g.Plan()
    assert p.passes["class"][0] == "dem" and len(p.passes["class"][1]) == 3
    assert len(p.passes["slope"][1]) == 1
    stages = p._stages(p.passes["class"][1]).stages
    assert [s.op for s in stages] == [2, 12, 13]
    assert "terrain.Slope -> transfer.Lookup -> transfer.Reclass" in p.String()


def test_graph_rejects_what_is_not_one_pass():
    g = graph.New()
    dem = g.Input("dem")
    two = graph.FocalMean(graph.Slope(dem, terrain.SlopeOptions(CellSize=10)), focal.BoxOptions(Radius=2))
    g.Output("x", two)
    with pytest.raises(NotSupported):
        g.Plan()


def test_graph_checks_options_when_building():
    g = graph.New()
    dem = g.Input("dem")
    with pytest.raises(StrataPanic, match="terrain: CellSize must be positive"):
        graph.Slope(dem, terrain.SlopeOptions())
    with pytest.raises(StrataPanic, match="used twice"):
        g.Output("dem", dem)


def test_stats_arithmetic():
    s = engine.Stats(Cells=10, Ideal=80, KernelRead=60, KernelWritten=40, SourceRead=0, SinkWritten=0)
    assert s.Total() == 100 and s.Amplification() == 100 / 80 and s.BytesPerCell() == 10
    assert s.Halo(1) == 60 - 40
    s.Add(engine.Stats(Cells=1, Ideal=8))
    assert s.Cells == 11 and s.Ideal == 88


def test_raster_validate_and_window():
    r = NewFloat32(5, 4, np.arange(20, dtype=np.float32))
    r.valid = mask_from_bool(np.ones((4, 5), bool))
    w = r.Window(1, 1, 3, 2)
    assert w.width == 3 and w.valid_offset == 6 and float(w.data[0]) == 6.0
    assert (w.numpy() == np.array([[6, 7, 8], [11, 12, 13]], np.float32)).all()
    with pytest.raises(StrataPanic):
        r.Window(3, 3, 3, 3)
    with pytest.raises(StrataPanic, match="stride 2 is less than width 5"):
        Float32Raster(np.zeros(20, np.float32), 5, 4, 2).Validate()
    like = NewFloat32Like(r)
    assert like.valid is not None and like.stride == 5


def test_negative_options_panic_before_any_device_work():
    """engine: negative Options panic (internal/exec/process.go:116-118), and
    the check runs before the device is touched, so it holds without one."""
    r = NewFloat32(8, 8, np.zeros(64, np.float32))
    d = NewFloat32Like(r)
    import ctypes

    from strata_b200 import _lib

    st = terrain.slope_stage(terrain.SlopeOptions(CellSize=1))
    o = _lib.ExecOpts()
    o.tile_width = -1
    rc = _lib.lib().strata_process(None, st.c_array(), 1, None, 0, None, 0, ctypes.byref(o), None)
    assert rc == _lib.EINVAL and "nil context" in _lib.last_error()
