"""Batches: many device-resident rasters of mixed sizes and ops in one
CUDA-graph launch, with band heights from an autotuner.

    items = [batch.Item(terrain.slope_stage(opts), src, [dst]), ...]
    b = batch.Batch(items)          # plans, uploads descriptors, captures the graph
    b.run()                         # one graph launch (synchronous by default)

Each item is one pipeline over one raster, with strata_process's edge and
validity rules, so a raster's result is the same alone and in a batch.
A raster's work units are bands of rows (512 columns wide for the
marching kernels, a band of 512 column results for the separable focal
ops; the windowed focal ops use fixed tiles). The band height of each op
class comes from the Autotuner: it times the candidate heights on a probe
raster of the class once per device and caches the winner (in memory, and
in a JSON file when a path is given). An item's tile is (width, height):
the width is fixed by the kernel and not used, the height is the band.
"""
from __future__ import annotations

import ctypes
import json
import os
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib, engine
from .raster import Float32Raster, StrataPanic

# Candidate bands (rows per work unit), as (width, height) tiles whose
# width the kernels fix: short bands spread a raster over more blocks,
# tall ones re-read fewer halo rows per cell.
CANDIDATES: List[Tuple[int, int]] = [(512, 16), (512, 32), (512, 64), (512, 128), (512, 256)]


@dataclass
class Item:
    stages: engine.StageList
    src: Float32Raster
    dst: Sequence[Float32Raster]
    tile: Optional[Tuple[int, int]] = None  # None: the autotuner's choice for the class


def _class_key(st: engine.StageList) -> Tuple[int, int]:
    s = st.stages[0]
    r = 1 if s.op in (_lib.OP_GRADIENT, _lib.OP_SLOPE, _lib.OP_ASPECT, _lib.OP_HILLSHADE, _lib.OP_CURVATURE) \
        else s.radius
    return int(s.op), int(r)


class Batch:
    """A planned batch (strata_batch_create): run() replays its graph."""

    def __init__(self, items: Sequence[Item], device: int = 0, tuner: Optional["Autotuner"] = None):
        self.device = device
        self.items = list(items)
        c = engine.device_context(device)
        arr = (_lib.BatchItem * len(self.items))()
        self._keep = []
        for i, it in enumerate(self.items):
            st = it.stages.c_array()
            self._keep.append(st)
            self._keep.append(it.stages)
            arr[i].stages = ctypes.cast(st, ctypes.POINTER(_lib.Stage))
            arr[i].nstages = len(it.stages.stages)
            if tuner is not None and it.tile is None:
                tuner.register(it.stages)
            tile = it.tile or (tuner.shape(_class_key(it.stages)) if tuner else None)
            if tile:
                arr[i].tile_width, arr[i].tile_height = tile
            arr[i].src = engine.c_raster(it.src)
            for k, d in enumerate(it.dst):
                arr[i].dst[k] = engine.c_raster(d)
        p = ctypes.c_void_p()
        _lib.check(_lib.lib().strata_batch_create(c, arr, len(self.items), ctypes.byref(p)))
        self._h = p

    def run(self, stream=None, synchronize: bool = True) -> None:
        s = getattr(stream, "cuda_stream", stream) if stream is not None else None
        _lib.check(_lib.lib().strata_batch_run(self._h, s, 1 if synchronize else 0))

    def stats(self) -> Tuple[engine.Stats, int]:
        st = _lib.Stats()
        n = ctypes.c_int()
        _lib.check(_lib.lib().strata_batch_info(self._h, ctypes.byref(st), ctypes.byref(n)))
        return engine.Stats(st.cells, st.ideal, st.tiles, st.bands, st.source_read, st.sink_written,
                            st.kernel_read, st.kernel_written), n.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().strata_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Autotuner:
    """Picks each op class's band height by timing the candidates on a probe
    raster of the class (probe x probe cells, seeded), once per device;
    results are cached in memory and, with a path, in a JSON file keyed by
    the device name."""

    def __init__(self, path: Optional[str] = None, probe: int = 1024, reps: int = 3, device: int = 0):
        self.path = path
        self.probe = probe
        self.reps = reps
        self.device = device
        self._lock = threading.Lock()
        self._cache: Dict[str, List[int]] = {}
        self._factories: Dict[Tuple[int, int], engine.StageList] = {}
        self._devname = None
        if path and os.path.exists(path):
            try:
                self._cache = json.load(open(path))
            except Exception:
                self._cache = {}

    def _key(self, cls) -> str:
        if self._devname is None:
            import torch

            self._devname = torch.cuda.get_device_name(self.device).replace(" ", "_")
        return f"{self._devname}:{cls[0]}:{cls[1]}"

    def register(self, stages: engine.StageList) -> None:
        """Remembers a stage list of its class, to probe with."""
        self._factories.setdefault(_class_key(stages), stages)

    def shape(self, cls: Tuple[int, int]) -> Optional[Tuple[int, int]]:
        with self._lock:
            k = self._key(cls)
            if k in self._cache:
                return tuple(self._cache[k])
            stages = self._factories.get(cls)
            if stages is None:
                return None
            best = self._tune(stages)
            self._cache[k] = list(best)
            if self.path:
                os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
                with open(self.path, "w") as f:
                    json.dump(self._cache, f, indent=1, sort_keys=True)
            return best

    def _tune(self, stages: engine.StageList) -> Tuple[int, int]:
        import torch

        from . import synth

        n = self.probe
        dev = torch.device("cuda", self.device)
        cells = torch.from_numpy(synth.fbm_dem(n, n, 0x7E57)).reshape(-1).to(dev)
        src = Float32Raster(cells, n, n, n)
        outs = [Float32Raster(torch.empty(n * n, dtype=torch.float32, device=dev), n, n, n) for _ in range(2)]
        nout = 2 if stages.stages[0].op == _lib.OP_GRADIENT else 1
        best, best_t = CANDIDATES[0], float("inf")
        for tile in CANDIDATES:
            try:
                b = Batch([Item(stages, src, outs[:nout], tile)], self.device)
            except StrataPanic:
                continue
            b.run()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(self.reps):
                b.run(synchronize=False)
            torch.cuda.synchronize()
            t = (time.perf_counter() - t0) / self.reps
            b.close()
            if t < best_t:
                best, best_t = tile, t
        return best
