#!/usr/bin/env python
"""Benchmark of the raster-stencil path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload (terrain16k): the full terrain set on a 16384 x 16384
float32 DEM (1 GiB; seeded diamond-square fBm, H = 0.8, scaled to
0-3000 m; 2% NoData as random 8x8 blocks in the validity mask; CellSize
10): Gradient, Slope, Aspect, Hillshade (azimuth 315, altitude 45, z 1),
profile / plan / mean Curvature, TRI / TPI / roughness, and the fused
Slope -> Lookup (knots 0,5,10,20,30,40 deg) -> Reclass (5 classes) pass.
One step runs every op of the set once over the DEM, with the DEM and the
outputs resident in HBM. The inputs (1 GiB) are larger than L2, so no
flush is needed between steps.

Other workloads: slope2k (Slope on 2048 x 2048, CellSize 30), focal8k
(focal ops on 8192 x 8192, r = 1..8), batch512, serve40k, raw8k (chunked
raw float32 file to raw file, Slope on 8192 x 8192 with a fill value).

value: whole-job Mcells/s, output cells of every op per second (an op
with two outputs counts its cells once). e2e: the same metric through the
public API with host (page-locked) buffers, the host-to-device copy of
the DEM and the device-to-host copy of each result inside the timed
region. roofline: the op with the largest share of the step, its
algorithmic bytes per launch over its average CUDA-event duration, against
the measured HBM copy bandwidth. cpu_baseline: the parity oracle (a C
restatement of the reference's scalar kernels) timed on the host cores on
a row band of the same DEM.

--impl reference times the reference's CPU implementation of the path:
the reference (Go) cannot be built here, so it is the oracle port, on all
host cores, each step a bounded row band of the workload.

Multi-GPU (under torchrun): each rank runs the whole workload on its own
GPU over its own DEM (independent rasters, no collective on the data
path); value is the cells of all ranks over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
SLOPE_XS, SLOPE_YS = [0, 5, 10, 20, 30, 40], [1, 1.1, 1.3, 1.9, 3, 4.5]
BREAKS, VALUES = [1.2, 1.6, 2.2, 3], [1, 2, 3, 4, 5]


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# Workloads: (name, stage-list factory, outputs) per op, and the input.

def _synth():
    """The synthetic-input generators (strata_b200/synth.py, numpy only),
    loaded by file so that the reference arm never imports the device
    package or maps its library."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("strata_synth", os.path.join(ROOT, "strata_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _orc():
    from oracle import oracle as orc

    return orc


# Each op of a workload: (name, device stages factory, oracle stages factory,
# outputs). The oracle factories resolve the same options with the oracle's
# own code (oracle/oracle.py), so the CPU legs load no device library.

def terrain_ops(cell_size):
    cs = cell_size

    def dev(fn):
        def mk():
            from strata_b200 import terrain, transfer  # noqa: F401

            return fn(terrain, transfer)
        return mk

    o = dict(CellSize=cs)
    return [
        ("gradient", dev(lambda t, _x: t.gradient_stage(t.GradientOptions(**o))),
         lambda: [_orc().gradient_stage(cs)], 2),
        ("slope", dev(lambda t, _x: t.slope_stage(t.SlopeOptions(**o))), lambda: [_orc().slope_stage(cs)], 1),
        ("aspect", dev(lambda t, _x: t.aspect_stage(t.AspectOptions(**o))), lambda: [_orc().aspect_stage(cs)], 1),
        ("hillshade", dev(lambda t, _x: t.hillshade_stage(t.HillshadeOptions(Azimuth=315, Altitude=45, ZFactor=1, **o))),
         lambda: [_orc().hillshade_stage(cs, azimuth=315, altitude=45)], 1),
        ("curvature_profile", dev(lambda t, _x: t.curvature_stage(t.CurvatureOptions(Type=0, **o))),
         lambda: [_orc().curvature_stage(cs, kind=0)], 1),
        ("curvature_plan", dev(lambda t, _x: t.curvature_stage(t.CurvatureOptions(Type=1, **o))),
         lambda: [_orc().curvature_stage(cs, kind=1)], 1),
        ("curvature_mean", dev(lambda t, _x: t.curvature_stage(t.CurvatureOptions(Type=2, **o))),
         lambda: [_orc().curvature_stage(cs, kind=2)], 1),
        ("tri", dev(lambda t, _x: t.ruggedness_stage(t.RuggednessOptions(Type=0, Radius=1))),
         lambda: [_orc().ruggedness_stage(0, 1)], 1),
        ("tpi", dev(lambda t, _x: t.ruggedness_stage(t.RuggednessOptions(Type=2, Radius=1))),
         lambda: [_orc().ruggedness_stage(2, 1)], 1),
        ("roughness", dev(lambda t, _x: t.ruggedness_stage(t.RuggednessOptions(Type=3, Radius=1))),
         lambda: [_orc().ruggedness_stage(3, 1)], 1),
        ("slope_lookup_reclass",
         dev(lambda t, x: t.slope_stage(t.SlopeOptions(**o)).extend(x.lookup_stage(SLOPE_XS, SLOPE_YS))
             .extend(x.reclass_stage(BREAKS, VALUES))),
         lambda: [_orc().slope_stage(cs), _orc().lookup_stage(SLOPE_XS, SLOPE_YS), _orc().reclass_stage(BREAKS, VALUES)],
         1),
    ]


def focal_ops():
    synth = _synth()
    ops = []
    for r in range(1, 9):
        w = synth.uniform_weights((2 * r + 1) ** 2, 0x5EED0003 + r)

        def dev(w=w, r=r):
            from strata_b200 import focal

            return focal.weights_stage(focal.WeightsOptions(r, w), False)

        ops.append((f"correlate_r{r}", dev, lambda w=w, r=r: [_orc().stage(_orc().CORRELATE, r, 0, (), [w])], 1))

    def gdev():
        from strata_b200 import focal

        g = focal.Gaussian(8, 2.5)
        return focal.separable_stage(focal.SeparableOptions(8, g, g))

    def gorc():
        g = _orc().gaussian(8, 2.5)
        return [_orc().stage(_orc().SEPARABLE, 8, 0, (), [g, g])]

    ops.append(("gaussian_r8", gdev, gorc, 1))
    for r in (3, 8):
        for name, code in (("mean", 9), ("min", 10), ("max", 11)):
            def dev(r=r, code=code):
                from strata_b200 import focal

                return focal.box_stage(focal.BoxOptions(r), code)

            ops.append((f"{name}_r{r}", dev, lambda r=r, code=code: [_orc().stage(code, r)], 1))
    return ops


def workload(name, side=None, only=None):
    """The named workload; side and only (profiling aids) replace its raster
    side and keep the named ops of its set."""
    wl = _workload(name, side)
    if only:
        keep = set(only.split(","))
        wl["ops"] = [o for o in wl["ops"] if o[0] in keep]
        if not wl["ops"]:
            raise SystemExit(f"no op of {name} is named in {only}")
    return wl


def _workload(name, side=None):
    synth = _synth()

    def slope_op(cs):
        def dev():
            from strata_b200 import terrain

            return terrain.slope_stage(terrain.SlopeOptions(CellSize=cs))
        return [("slope", dev, lambda: [_orc().slope_stage(cs)], 1)]

    if name == "terrain16k":
        n, seed, cs = side or 16384, 0x5EED0002, 10
        cells = synth.fbm_dem(n, n, seed)
        valid = synth.block_mask(n, n, seed, 0.02)
        return dict(name=f"terrain set on {n}x{n} f32 DEM", width=n, height=n, cells=cells, valid=valid,
                    ops=terrain_ops(cs), cell_size=cs, mask="2% NoData in 8x8 blocks", radius=1)
    if name in ("slope2k", "slope8k"):
        n, seed, cs = side or (2048 if name == "slope2k" else 8192), 0x5EED0001, 30
        return dict(name=f"Slope on {n}x{n} f32 DEM", width=n, height=n, cells=synth.fbm_dem(n, n, seed),
                    valid=synth.block_mask(n, n, seed, 0.02), cell_size=cs, mask="2% NoData in 8x8 blocks",
                    ops=slope_op(cs), radius=1)
    if name == "pipeline8k":
        n, seed, cs = side or 8192, 0x5EED0002, 10
        ops = [o for o in terrain_ops(cs) if o[0] == "slope_lookup_reclass"]
        return dict(name=f"Slope->Lookup->Reclass on {n}x{n} f32 DEM", width=n, height=n,
                    cells=synth.fbm_dem(n, n, seed), valid=synth.block_mask(n, n, seed, 0.02), cell_size=cs,
                    mask="2% NoData in 8x8 blocks", ops=ops, radius=1)
    if name == "focal8k":
        n, seed = side or 8192, 0x5EED0003
        return dict(name=f"focal ops on {n}x{n} f32 raster", width=n, height=n, cells=synth.normal_trend(n, n, seed),
                    valid=synth.cell_mask(n, n, seed, 0.05), ops=focal_ops(), cell_size=None,
                    mask="5% random NoData cells", radius=8)
    raise SystemExit(f"unknown workload {name}")


def alg_bytes(cells, nout, masked):
    """Algorithmic bytes of one op over `cells` cells: one input read and
    nout outputs written, 4 B a cell, plus 1/8 B a cell per mask."""
    b = cells * 4 * (1 + nout)
    if masked:
        b += cells * (1 + nout) / 8.0
    return b


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.

class Clocks:
    def __init__(self, index):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# The CPU legs, on the oracle only (oracle/: the scalar restatement of the
# reference's kernels and, with simd, the restated AVX2 lanes of the
# reference's internal/stencil/simd_amd64.go).

def _band(wl, y0, y1):
    """Rows [y0, y1) of the workload's input as an oracle raster (a raster
    of its own: its first and last rows are its edge ring)."""
    orc = _orc()
    W = wl["width"]
    cells = np.ascontiguousarray(wl["cells"][y0:y1])
    valid = wl["valid"][y0:y1] if wl["valid"] is not None else None
    return dict(data=cells.reshape(-1), width=W, height=y1 - y0, stride=W,
                valid=orc.pack_mask(valid) if valid is not None else None, valid_offset=0)


def _outs(src, n):
    cells = src["width"] * src["height"]
    return [dict(data=np.empty(cells, np.float32), width=src["width"], height=src["height"], stride=src["width"],
                 valid=np.zeros((cells + 63) // 64, np.uint64) if src["valid"] is not None else None, valid_offset=0)
            for _ in range(n)]


def cpu_run(wl, src, nthreads, simd, reps=1):
    """Every op of the workload with the oracle over the raster src;
    returns (output cells, seconds)."""
    orc = _orc()
    outs = _outs(src, 2)
    stages = [(mk(), nout) for _n, _d, mk, nout in wl["ops"]]
    total, t0 = 0, time.perf_counter()
    for _ in range(reps):
        for st, nout in stages:
            orc.process(st, src, outs[:nout], nthreads, simd=simd)
            total += src["width"] * src["height"]
    return total, time.perf_counter() - t0


def cpu_baseline(wl, target_s=12.0):
    """The restated AVX2 path on every host core over a bounded row band of
    the workload (every op of the set), and the scalar oracle on one
    thread beside it."""
    threads = os.cpu_count() or 1
    rows = min(wl["height"], max(64, (1 << 24) // wl["width"]))
    src = _band(wl, 0, rows)
    cells, secs = cpu_run(wl, src, threads, True)
    reps = max(1, int(target_s / max(secs, 1e-3)))
    cells, secs = cpu_run(wl, src, threads, True, reps)
    srows = max(8, rows // 16)
    s1 = _band(wl, 0, srows)
    c1, t1 = cpu_run(wl, s1, 1, False)
    return {"value": round(cells / secs / 1e6, 1), "unit": "Mcells/s", "cores": threads, "kind": "restated-avx2",
            "sample": f"{rows} rows x {wl['width']} cells of the workload, every op of the set, {reps} pass(es), "
                      f"{secs:.1f} s; AVX2 lanes after internal/stencil/simd_amd64.go (radius-1 stencils), "
                      f"the scalar kernels elsewhere",
            "scalar_1thread": {"value": round(c1 / t1 / 1e6, 1), "unit": "Mcells/s", "cores": 1,
                               "sample": f"{srows} rows x {wl['width']} cells, every op, scalar oracle"}}


def parity_check(wl, fetch):
    """The device's outputs against the oracle on two row bands of the
    workload (its first rows, with the raster's top edge, and rows in the
    middle): fetch(i, y0, y1) returns op i's output rows [y0, y1) as (data
    rows, validity rows as bools or None), for each output. Each band runs
    through the oracle as a raster of its own, so the band's interior rows
    (the radius in from a band edge that is not the raster's) are compared,
    every cell (rastertest.SameFloat: same bits, or both NaN) and every
    validity bit."""
    orc = _orc()
    H, W, r = wl["height"], wl["width"], wl["radius"]
    band = min(H, 64 + 2 * r)
    mid = max(0, H // 2 - band // 2)
    checked = cells = bad = vbad = 0
    for i, (_name, _dev, mk, nout) in enumerate(wl["ops"]):
        for y0 in sorted({0, mid}):
            y1 = min(H, y0 + band)
            src = _band(wl, y0, y1)
            want = _outs(src, nout)
            orc.process(mk(), src, want, os.cpu_count() or 1, simd=False)
            lo = 0 if y0 == 0 else r
            hi = (y1 - y0) if y1 == H else (y1 - y0) - r
            got = fetch(i, y0, y1)
            for k in range(nout):
                g = got[k][0][lo:hi]
                w = want[k]["data"].reshape(y1 - y0, W)[lo:hi]
                same = (g.view(np.uint32) == w.view(np.uint32)) | (np.isnan(g) & np.isnan(w))
                bad += int((~same).sum())
                cells += same.size
                if want[k]["valid"] is not None:
                    wv = np.unpackbits(want[k]["valid"].view(np.uint8), bitorder="little")[:(y1 - y0) * W]
                    wv = wv.reshape(y1 - y0, W)[lo:hi].astype(bool)
                    vbad += int((got[k][1][lo:hi] != wv).sum())
        checked += 1
    return {"ops_checked": checked, "cells": cells, "mismatches": bad, "validity_mismatches": vbad,
            "bands": f"rows 0..{band} and {mid}..{mid + band}, interior rows compared", "oracle": "scalar"}


# ---------------------------------------------------------------------------
# Our arm.

def run_ours(args, rank, world, local_rank):
    import torch

    from strata_b200 import engine
    from strata_b200.raster import Float32Raster, mask_from_bool

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = workload(args.workload, args.side, args.ops)
    W, H = wl["width"], wl["height"]
    n = W * H
    masked = wl["valid"] is not None
    host_cells = torch.from_numpy(wl["cells"].reshape(-1)).pin_memory()
    host_mask = torch.from_numpy(mask_from_bool(wl["valid"]).view(np.int64)).pin_memory()
    src = Float32Raster(host_cells.to(dev), W, H, W, host_mask.to(dev), 0)
    words = (n + 63) // 64
    outs = [Float32Raster(torch.empty(n, dtype=torch.float32, device=dev), W, H, W,
                          torch.empty(words, dtype=torch.int64, device=dev), 0) for _ in range(2)]
    stream = torch.cuda.Stream(dev)
    opts = engine.Options(Stream=stream, Async=True, Device=local_rank)
    ops = [(name, dev(), nout) for name, dev, _mk, nout in wl["ops"]]
    n_outs = sum(nout for _n, _s, nout in ops)
    # Every output of the set, device-resident: the timed step is one
    # terrain.Features call over the set (engine.process_features), which
    # runs the memory-bound radius-1 ops as one fused pass over the input
    # and the others as their own launches.
    all_outs = [Float32Raster(torch.empty(n, dtype=torch.float32, device=dev), W, H, W,
                              torch.empty(words, dtype=torch.int64, device=dev), 0) for _ in range(n_outs)]
    feats = [st for _n, st, _o in ops]

    def step():
        assert engine.process_features(feats, all_outs, src, opts) is None

    def separate(events=None):
        for i, (name, stages, nout) in enumerate(ops):
            if events is not None:
                events[i][0].record(stream)
            err = engine.process(stages, outs[:nout], [src], opts)
            assert err is None
            if events is not None:
                events[i][1].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
            separate()
    torch.cuda.synchronize()

    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()

    per_op = [[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] for _ in ops]
    op_ms = [0.0] * len(ops)
    # Per-op durations, each op run alone (engine.process): K back-to-back
    # calls of the op between two events, after one untimed call that keeps
    # the stream busy while the host issues the timed ones (so no host issue
    # time lands inside the events).
    with torch.cuda.stream(stream):
        for i, (name, stages, nout) in enumerate(ops):
            assert engine.process(stages, outs[:nout], [src], opts) is None
            per_op[i][0].record(stream)
            for _ in range(args.steps):
                assert engine.process(stages, outs[:nout], [src], opts) is None
            per_op[i][1].record(stream)
        torch.cuda.synchronize()
        for i in range(len(ops)):
            op_ms[i] = per_op[i][0].elapsed_time(per_op[i][1]) / args.steps

    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                step()
            end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.steps
    barrier()
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    cells_per_step = n * len(ops)
    value = world * cells_per_step / (ms / 1e3) / 1e6
    peak, peak_kind = hbm_peak()
    per = []
    for i, (name, _st, nout) in enumerate(ops):
        b = alg_bytes(n, nout, masked)
        gbs = b / (op_ms[i] / 1e3) / 1e9
        per.append({"op": name, "ms": round(op_ms[i], 4), "mcells_s": round(n / (op_ms[i] / 1e3) / 1e6, 1),
                    "gbs": round(gbs, 1), "frac_hbm": round(gbs / peak, 4)})
    traffic_db = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic_db = json.load(open(tpath)).get(args.workload, {})
        except Exception:
            traffic_db = {}
    fused = [i for i, (_nm, st, _o) in enumerate(ops) if _fusable(st)]
    firsts = np.cumsum([0] + [nout for _n, _s, nout in ops])
    fused_ms = None
    if len(fused) >= 2:
        # The fused pass alone (the step's one kernel for those features).
        f_outs = [all_outs[int(firsts[i]) + k] for i in fused for k in range(ops[i][2])]
        f_feats = [ops[i][1] for i in fused]
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            assert engine.process_features(f_feats, f_outs, src, opts) is None
            ev0.record(stream)
            for _ in range(args.steps):
                assert engine.process_features(f_feats, f_outs, src, opts) is None
            ev1.record(stream)
        torch.cuda.synchronize()
        fused_ms = ev0.elapsed_time(ev1) / args.steps
    # The step's kernels: the fused pass, and each other op's own launch.
    kernels = [(ops[i][0], op_ms[i], alg_bytes(n, ops[i][2], masked)) for i in range(len(ops))
               if fused_ms is None or i not in fused]
    if fused_ms is not None:
        f_nout = sum(ops[i][2] for i in fused)
        kernels.append((f"features_tma_kernel (the fused pass: {', '.join(ops[i][0] for i in fused)})", fused_ms,
                        n * 4 * (1 + f_nout) + (n * (1 + f_nout) / 8.0 if masked else 0)))
    kname, kms, top_bytes = max(kernels, key=lambda k: k[1])
    achieved = top_bytes / (kms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic_db.get("features" if kname.startswith("features_tma") else kname),
                "alg_bytes_per_launch": int(top_bytes), "ms": round(kms, 4)}
    launches_per_step = len(kernels)
    fused_line = None
    if fused_ms is not None:
        fb = kernels[-1][2]
        fused_line = {"ops": [ops[i][0] for i in fused], "ms": round(fused_ms, 4),
                      "separate_ms": round(sum(op_ms[i] for i in fused), 4),
                      "gbs": round(fb / (fused_ms / 1e3) / 1e9, 1),
                      "frac_hbm": round(fb / (fused_ms / 1e3) / 1e9 / peak, 4)}
    separate_ms = sum(op_ms)

    # Parity at the benchmarked size: the timed call's outputs (every op of
    # the set from one Features call), two row bands of each against the
    # oracle on the same rows.
    with torch.cuda.stream(stream):
        step()
    torch.cuda.synchronize()

    def fetch(i, y0, y1):
        res = []
        for k in range(ops[i][2]):
            o = all_outs[int(firsts[i]) + k]
            d = o.data[y0 * W:y1 * W].cpu().numpy().reshape(y1 - y0, W)
            b0, b1 = y0 * W, y1 * W
            wd = o.valid[b0 // 64:(b1 + 63) // 64].cpu().numpy().view(np.uint8)
            bits = np.unpackbits(wd, bitorder="little")[b0 - (b0 // 64) * 64:][:b1 - b0]
            res.append((d, bits.reshape(y1 - y0, W).astype(bool)))
        return res

    parity = parity_check(wl, fetch) if rank == 0 else None

    # e2e: the public API with host (page-locked) buffers, every copy inside
    # the timed region: one process_features call (terrain.Features) for
    # every op of the set, the pipeline included, so the DEM crosses once
    # and each output's copy back overlaps the next op's kernels.
    host_src = Float32Raster(host_cells.numpy(), W, H, W, host_mask.numpy().view(np.uint64), 0)
    del all_outs
    host_outs = [Float32Raster(torch.empty(n, dtype=torch.float32).pin_memory().numpy(), W, H, W,
                               torch.zeros(words, dtype=torch.int64).pin_memory().numpy().view(np.uint64), 0)
                 for _ in range(n_outs)]
    e2e_opts = engine.Options(Device=local_rank)

    def e2e_step():
        assert engine.process_features([st for _n, st, _o in ops], host_outs, host_src, e2e_opts) is None

    e2e_step()
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    barrier()
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = n * 4 + words * 8
    d2h = n_outs * (n * 4 + words * 8)
    e2e = {"value": round(world * cells_per_step / e2e_s / 1e6, 1), "unit": "Mcells/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_s * 1e3, 2),
           "api": "engine.process_features (terrain.Features) over every op, host rasters"}


    line = {
        "metric": "Mcells/s (output cells of every op in the set per second)", "value": round(value, 1),
        "unit": "Mcells/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl["name"], "width": W, "height": H, "cell_size": wl["cell_size"],
                   "ops": [o[0] for o in ops], "mask": wl["mask"], "l2": "inputs larger than L2 (no flush)",
                   "parallelism": f"independent rasters x{world}"},
        "roofline": roofline, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(), "per_op": per, "parity": parity,
        "fused_pass": fused_line,
        "separate_calls": {"value": round(world * cells_per_step / (separate_ms / 1e3) / 1e6, 1), "unit": "Mcells/s",
                           "ms_per_step": round(separate_ms, 4),
                           "api": "engine.process per op (each op alone, its own read of the input)"},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl)
    return line


def batch_rasters(seed=0x5EED0004, count=512):
    """The batched workload: `count` rasters with width and height each
    log-uniform in 64..4096 (windows of one seeded fBm mosaic, so each is
    fBm terrain), 2% NoData in 8x8 blocks, each with one op from {Slope,
    Hillshade, Curvature (kind uniform), Correlate r in 1..8 (uniform
    [-1, 1] weights)} and CellSize uniform in 1..90."""
    from strata_b200 import focal, synth, terrain

    rng = np.random.default_rng(seed)
    mosaic = synth.fbm_dem(8192, 8192, seed)
    out = []
    for i in range(count):
        w = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
        h = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
        x = int(rng.integers(0, 8192 - w + 1))
        y = int(rng.integers(0, 8192 - h + 1))
        cells = np.ascontiguousarray(mosaic[y:y + h, x:x + w])
        valid = synth.block_mask(w, h, seed + i, 0.02)
        cs = float(rng.uniform(1, 90))
        kind = int(rng.integers(4))
        if kind == 0:
            name, st = "slope", terrain.slope_stage(terrain.SlopeOptions(CellSize=cs))
        elif kind == 1:
            name, st = "hillshade", terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=cs))
        elif kind == 2:
            t = int(rng.integers(3))
            name, st = f"curvature{t}", terrain.curvature_stage(terrain.CurvatureOptions(CellSize=cs, Type=t))
        else:
            r = int(rng.integers(1, 9))
            wts = synth.uniform_weights((2 * r + 1) ** 2, seed + 7 * i)
            name, st = f"correlate_r{r}", focal.weights_stage(focal.WeightsOptions(r, wts), False)
        out.append((name, st, cells, valid))
    return out


def run_batch(args, rank, world, local_rank):
    """The batched form against per-raster plain launches, same rasters."""
    import torch

    from strata_b200 import batch, engine
    from strata_b200.raster import Float32Raster, mask_from_bool

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    rasters = batch_rasters()
    items, cells = [], 0
    for name, st, c, v in rasters:
        h, w = c.shape
        n = w * h
        words = (n + 63) // 64
        src = Float32Raster(torch.from_numpy(c.reshape(-1)).to(dev), w, h, w,
                            torch.from_numpy(mask_from_bool(v).view(np.int64)).to(dev), 0)
        dst = Float32Raster(torch.empty(n, dtype=torch.float32, device=dev), w, h, w,
                            torch.empty(words, dtype=torch.int64, device=dev), 0)
        items.append(batch.Item(st, src, [dst]))
        cells += n
    tuner = batch.Autotuner(path=os.path.join(ROOT, "strata_b200", "tuning.json") if args.tune_cache else None)
    b = batch.Batch(items, local_rank, tuner)
    opts = engine.Options(Device=local_rank)

    def plain_step():
        for it in items:
            assert engine.process(it.stages, it.dst, [it.src], opts) is None

    for _ in range(args.warmup):
        b.run()
        plain_step()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.Stream(dev)  # the graph runs on this stream, which the events time
    with Clocks(local_rank) as clk:
        start.record(stream)
        for _ in range(args.steps):
            b.run(stream=stream, synchronize=False)
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.steps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        plain_step()
    torch.cuda.synchronize()
    plain_ms = (time.perf_counter() - t0) / args.steps * 1e3
    st, classes = b.stats()
    # Parity: a sample of the batch's rasters (every 32nd, up to 2^20 cells
    # each) against the oracle on the same raster, every cell and bit.
    orc = _orc()
    pbad = pv = pcells = pn = 0
    for i in range(0, len(items), 32):
        name, stg, c, v = rasters[i]
        h, w = c.shape
        if w * h > (1 << 20):
            continue
        src = dict(data=np.ascontiguousarray(c.reshape(-1)), width=w, height=h, stride=w,
                   valid=orc.pack_mask(v), valid_offset=0)
        want = _outs(src, 1)
        orc.process([_orc_of(x) for x in stg.stages], src, want, os.cpu_count() or 1)
        g = items[i].dst[0].data.cpu().numpy()
        wv = np.unpackbits(want[0]["valid"].view(np.uint8), bitorder="little")[:w * h].astype(bool)
        gv = np.unpackbits(items[i].dst[0].valid.cpu().numpy().view(np.uint8), bitorder="little")[:w * h].astype(bool)
        same = (g.view(np.uint32) == want[0]["data"].view(np.uint32)) | (np.isnan(g) & np.isnan(want[0]["data"]))
        pbad += int((~same).sum())
        pv += int((gv != wv).sum())
        pcells += w * h
        pn += 1
    value = world * cells / (ms / 1e3) / 1e6
    plain = world * cells / (plain_ms / 1e3) / 1e6
    peak, peak_kind = hbm_peak()
    alg = sum(alg_bytes(it.src.width * it.src.height, 1, True) for it in items)
    line = {
        "metric": "Mcells/s (batched rasters, one graph launch)", "value": round(value, 1), "unit": "Mcells/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch of 512 rasters, sides log-uniform 64..4096, mixed ops", "rasters": len(items),
                   "cells": cells, "classes": classes, "l2": "inputs larger than L2 (no flush)"},
        "plain_launches": {"value": round(plain, 1), "unit": "Mcells/s", "ms_per_step": round(plain_ms, 3),
                           "api": "engine.process per raster, synchronous"},
        "batched_over_plain": round(plain_ms / ms, 2),
        "roofline": {"bound": "hbm", "kernel": "batch_kernel (all classes)", "achieved": round(alg / (ms / 1e3) / 1e9, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(alg / (ms / 1e3) / 1e9 / peak, 4), "traffic": None},
        "gpu_launches": classes * args.steps, "clocks": clk.summary(),
        "parity": {"rasters_checked": pn, "cells": pcells, "mismatches": pbad, "validity_mismatches": pv,
                   "sample": "every 32nd raster of at most 2^20 cells, against the scalar oracle"},
    }
    b.close()
    return line


def serve_mosaic(n, seed, dev):
    """A 40000 x 40000 (n x n) DEM resident on the device: a 4096 x 4096
    diamond-square fBm tile, mirrored into a seamless 8192 period and tiled,
    plus a gentle trend; 2% NoData as random 8x8 blocks."""
    import torch

    from strata_b200 import synth
    from strata_b200.raster import Float32Raster

    t = torch.from_numpy(synth.fbm_dem(4096, 4096, seed)).to(dev)
    t = torch.cat([torch.cat([t, t.flip(1)], 1), torch.cat([t.flip(0), t.flip(0).flip(1)], 1)], 0)
    reps = (n + 8191) // 8192
    cells = t.repeat(reps, reps)[:n, :n].contiguous()
    del t
    for y0 in range(0, n, 4096):  # the trend, a band at a time
        ys = torch.arange(y0, min(n, y0 + 4096), device=dev, dtype=torch.float32)[:, None]
        cells[y0:y0 + ys.shape[0]] += 0.002 * (ys + torch.arange(n, device=dev, dtype=torch.float32)[None, :])
    valid = torch.ones((n, n), dtype=torch.bool, device=dev)
    g = torch.Generator(device="cpu").manual_seed(seed)
    nblocks = -(-int(0.02 * n * n) // 64)
    bx = torch.randint(0, n - 8, (nblocks,), generator=g).to(dev)
    by = torch.randint(0, n - 8, (nblocks,), generator=g).to(dev)
    for dy in range(8):
        for dx in range(8):
            valid[by + dy, bx + dx] = False
    flat = valid.reshape(-1)
    words = (flat.numel() + 63) // 64
    pad = torch.ones(words * 64 - flat.numel(), dtype=torch.bool, device=dev)
    bits = torch.cat([flat, pad]).reshape(words, 64)
    del valid, flat
    w = torch.zeros(words, dtype=torch.int64, device=dev)
    for j in range(64):  # bit j of word i is cell 64 i + j
        w |= bits[:, j].to(torch.int64) << j
    del bits
    return Float32Raster(cells.reshape(-1), n, n, n, w, 0)


def run_serve(args, rank, world, local_rank):
    """Serving: window requests over a resident mosaic, batched as they
    arrive (continuous batching), against the same requests run one at a
    time through engine.process."""
    import torch

    from strata_b200 import engine, focal, serve, terrain
    from strata_b200.raster import Float32Raster

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n, seed = 40000, 0x5EED0005
    mosaic = serve_mosaic(n, seed, dev)
    ops = [("slope", terrain.slope_stage(terrain.SlopeOptions(CellSize=30))),
           ("aspect", terrain.aspect_stage(terrain.AspectOptions(CellSize=30))),
           ("hillshade", terrain.hillshade_stage(terrain.HillshadeOptions(CellSize=30))),
           ("mean_r5", focal.box_stage(focal.BoxOptions(Radius=5), engine._lib.OP_MEAN)),
           ("tpi", terrain.ruggedness_stage(terrain.RuggednessOptions(Type=terrain.RuggednessTPI)))]
    rng = np.random.default_rng(seed)
    per_step = 256

    def requests(k):
        out = []
        for _ in range(k):
            w = int(np.exp(rng.uniform(np.log(256), np.log(4096))))
            h = int(np.exp(rng.uniform(np.log(256), np.log(4096))))
            out.append((int(rng.integers(len(ops))), int(rng.integers(0, n - w + 1)), int(rng.integers(0, n - h + 1)),
                        w, h))
        return out

    srv = serve.Server(mosaic, budget_bytes=120 << 30, streams=4, max_batch=64, device=local_rank,
                       band=args.band or 0)

    def burst(reqs):
        """All at once (closed loop, the requests submitted, waited for and
        released as one group each): served cells over the wall time."""
        t0 = time.perf_counter()
        tickets = srv.submit_many([(ops[o][1], x, y, w, h) for o, x, y, w, h in reqs])
        srv.wait_many(tickets)
        srv.release_many(tickets)
        return sum(w * h for _o, _x, _y, w, h in reqs) / (time.perf_counter() - t0)

    for _ in range(args.warmup):
        burst(requests(per_step))
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        rates = [burst(requests(per_step)) for _ in range(args.steps)]
    capacity = statistics.median(rates)

    # Open loop: Poisson arrivals at 60% of that capacity.
    reqs = requests(per_step * args.steps)
    mean_cells = float(np.mean([w * h for _o, _x, _y, w, h in reqs]))
    rate = 0.6 * capacity / mean_cells  # requests per second
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, len(reqs))
    due = np.cumsum(gaps)
    # One thread submits the requests whose arrival time has come (one
    # submit_many call for all that are due); another waits for and
    # releases them in order (wait_many / release_many), so the client keeps
    # up with the offered load. The latencies are the server's own
    # submit-to-done times, so waiting late does not lengthen them.
    import queue
    import threading

    lat = []
    issued = queue.Queue()
    failed = []

    def drain():
        done = False
        while not done:
            batch = []
            t = issued.get()
            while True:
                if t is None:
                    done = True
                    break
                batch.append(t)
                if len(batch) >= 256 or issued.empty():
                    break
                t = issued.get()
            if batch and not failed:
                try:
                    lat.extend(r.latency_ms for r in srv.wait_many(batch))
                    srv.release_many(batch)
                except Exception as e:  # kept, and raised after the join
                    failed.append(e)

    drainer = threading.Thread(target=drain)
    drainer.start()
    nxt = 0
    t0 = time.perf_counter()
    while nxt < len(reqs):
        now = time.perf_counter() - t0
        k = nxt
        while k < len(reqs) and due[k] <= now:
            k += 1
        if k > nxt:
            for t in srv.submit_many([(ops[o][1], x, y, w, h) for o, x, y, w, h in reqs[nxt:k]]):
                issued.put(t)
            nxt = k
        elif due[nxt] - now > 2e-4:
            time.sleep(1e-4)
    issued.put(None)
    drainer.join()
    open_s = time.perf_counter() - t0
    if failed:
        raise failed[0]
    assert len(lat) == len(reqs), f"{len(lat)} latencies for {len(reqs)} requests"
    st = srv.stats()
    srv.close()

    # The same requests one at a time, synchronously, through engine.process.
    plain_reqs = reqs[:per_step]
    opts = engine.Options(Device=local_rank)
    outs = {}

    def plain():
        t1 = time.perf_counter()
        for o, x, y, w, h in plain_reqs:
            if (w, h) not in outs:
                outs[(w, h)] = Float32Raster(torch.empty(w * h, dtype=torch.float32, device=dev), w, h, w,
                                             torch.empty((w * h + 63) // 64, dtype=torch.int64, device=dev), 0)
            assert engine.process(ops[o][1], [outs[(w, h)]], [mosaic.Window(x, y, w, h)], opts) is None
        torch.cuda.synchronize()
        return sum(w * h for _o, _x, _y, w, h in plain_reqs) / (time.perf_counter() - t1)

    plain()
    plain_rate = plain()
    line = {
        "metric": "Mcells/s served (window requests over a resident mosaic, continuous batching)",
        "value": round(world * capacity / 1e6, 1), "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(per_step * mean_cells / capacity * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "40000x40000 resident DEM mosaic (fBm tile mirrored and tiled, 2% NoData 8x8 blocks), "
                               "windows with sides log-uniform 256..4096 at uniform origins, "
                               "ops Slope/Aspect/Hillshade/Mean r5/TPI", "requests_per_step": per_step,
                   "budget_bytes": 120 << 30, "streams": 4, "max_batch": 64, "band": args.band or "default",
                   "timing": "host wall clock (the serving path is asynchronous)",
                   "closed_loop": "value: each step's requests submitted, waited for and released as one group"},
        "latency_ms": {"offered_load": "Poisson arrivals at 60% of the closed-loop capacity",
                       "client": "one thread submits the due requests (submit_many), another waits for and "
                                 "releases them in order (wait_many, release_many)",
                       "requests": len(lat), "p50": round(float(np.percentile(lat, 50)), 3),
                       "p99": round(float(np.percentile(lat, 99)), 3), "mean": round(float(np.mean(lat)), 3),
                       "served_mcells_s": round(sum(w * h for _o, _x, _y, w, h in reqs) / open_s / 1e6, 1)},
        "plain_launches": {"value": round(plain_rate / 1e6, 1), "unit": "Mcells/s",
                           "api": "engine.process per window view, one at a time, synchronous"},
        "served_over_plain": round(capacity / plain_rate, 2),
        "server": st, "clocks": clk.summary(),
    }
    return line


def _fusable(stages):
    """Whether a feature runs in the fused multi-output pass (the library
    decides, features.cu; this mirrors it for the launch count): Gradient,
    Slope in percent or followed by a Reclass, and Wilson's TRI, TPI and
    roughness at radius 1."""
    st = stages.stages[0]
    tail = [x.op for x in stages.stages[1:]]
    folds = bool(tail) and tail[-1] == 13 and all(t in (12, 13) for t in tail)
    if tail and not folds:
        return False
    return (st.op == 1 or (st.op == 2 and (st.kind == 0 or folds)) or
            (st.op == 6 and st.radius == 1 and st.kind in (1, 2, 3)))


def _orc_of(st):
    """The oracle stage equal to one device stage (its op, radius, kind,
    constants and tables)."""
    import ctypes

    from strata_b200 import _lib

    tables = []
    for i in range(4):
        n = st.table_len[i]
        tables.append(np.ctypeslib.as_array((ctypes.c_float * n).from_address(st.table[i])).copy()
                      if st.table[i] and n > 0 else np.zeros(0, np.float32))
    while tables and tables[-1].size == 0:
        tables.pop()
    return _orc().stage(st.op, st.radius, st.kind, list(st.k), tables, flags=st.flags & _lib.STAGE_FIT,
                        input=st.input)


def run_raw(args, rank, world, local_rank):
    """Chunked raw file -> raw file (engine/raw.go, exec.ProcessChunked):
    Slope (CellSize 30) over a 8192 x 8192 little-endian float32 file whose
    NoData cells (2% in 8x8 blocks) hold the fill value -9999, into a file
    with fill -1 under invalid cells; full-width tiles of 1024 rows. Each
    step is one whole call (pread into page-locked memory, validity from
    the fill on the device, the stencil, the fill under invalid cells on
    the device, pwrite), timed by the wall clock around it since the host
    I/O is the work; the files sit in the page cache after the warm-up.
    The reference's figure for the same path is its chunked raw-to-raw
    Slope, 770-845 Mcells/s on 12 workers."""
    import shutil
    import tempfile

    from strata_b200 import engine, terrain

    synth = _synth()
    n = args.side or 8192
    seed, fill, out_fill = 0x5EED0001, np.float32(-9999), np.float32(-1)
    cells = synth.fbm_dem(n, n, seed)
    valid = synth.block_mask(n, n, seed, 0.02)
    cells = np.where(valid, cells, fill).astype("<f4")
    d = tempfile.mkdtemp(prefix="strata_raw_")
    try:
        sp, dp = os.path.join(d, "dem.f32"), os.path.join(d, "slope.f32")
        cells.tofile(sp)
        with open(dp, "wb") as g:
            g.truncate(4 * n * n)
        st = lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=30))
        opts = engine.Options(Device=local_rank, TileHeight=1024)
        with open(sp, "rb") as f, open(dp, "r+b") as g:
            src = engine.RawSource(f, n, n, engine.RawOptions(Fill=fill, HasFill=True))
            sink = engine.RawSink(g, n, n, engine.RawOptions(Fill=out_fill, HasFill=True))
            for _ in range(max(1, args.warmup)):
                assert engine.process_raw(st(), [sink], [src], opts) is None
            t0 = time.perf_counter()
            for _ in range(args.steps):
                assert engine.process_raw(st(), [sink], [src], opts) is None
            secs = time.perf_counter() - t0
        # parity: rows [0, 256] of the output against the oracle over rows
        # [0, 258) of the raster (whose own edge ring is its row 257)
        orc = _orc()
        rows = min(n, 258)
        band = dict(data=np.ascontiguousarray(cells[:rows]).reshape(-1).astype(np.float32), width=n, height=rows,
                    stride=n, valid=orc.pack_mask(valid[:rows]), valid_offset=0)
        out = _outs(band, 1)
        orc.process([orc.slope_stage(30)], band, out, os.cpu_count() or 1)
        want = out[0]["data"].reshape(rows, n).copy()
        vbits = np.unpackbits(out[0]["valid"].view(np.uint8), bitorder="little")[:rows * n].reshape(rows, n)
        want[vbits == 0] = out_fill
        got = np.fromfile(dp, "<f4", count=(rows - 1) * n).reshape(rows - 1, n)
        w2 = want[:rows - 1]
        bad = ~((got.view(np.uint32) == w2.view(np.uint32)) | (np.isnan(got) & np.isnan(w2)))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    value = n * n * args.steps / secs / 1e6
    return {"metric": "Mcells/s (chunked raw file to raw file, Slope)", "value": round(value, 1), "unit": "Mcells/s",
            "ms_per_step": round(secs / args.steps * 1e3, 2), "steps": args.steps,
            "config": {"workload": f"Slope, raw {n}x{n} f32 file -> raw file, fill -9999 (2% 8x8 blocks) -> -1",
                       "tiles": f"{n} x 1024", "clock": "wall (host I/O inside), files in the page cache"},
            "reference_published": {"value": "770-845", "unit": "Mcells/s", "workers": 12,
                                    "source": "the reference's chunked raw-to-raw Slope figure"},
            "parity": {"rows_checked": rows - 1, "cells": int(w2.size), "mismatches": int(bad.sum())}}


def run_stats(args, local_rank):
    """engine.Stats of each op of the workload, one plain call each over the
    device-resident raster, as JSON lines (op, cells, ideal, kernel_read,
    kernel_written in bytes): the byte counts an ncu capture of the same
    command sets beside dram__bytes_read.sum / dram__bytes_write.sum of the
    op's launches. No timing."""
    import torch

    from strata_b200 import engine
    from strata_b200.raster import Float32Raster, mask_from_bool

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = workload(args.workload, args.side, args.ops)
    W, H = wl["width"], wl["height"]
    n, words = W * H, (W * H + 63) // 64
    src = Float32Raster(torch.from_numpy(wl["cells"].reshape(-1)).to(dev), W, H, W,
                        torch.from_numpy(mask_from_bool(wl["valid"]).view(np.int64)).to(dev), 0)
    outs = [Float32Raster(torch.empty(n, dtype=torch.float32, device=dev), W, H, W,
                          torch.empty(words, dtype=torch.int64, device=dev), 0) for _ in range(2)]
    for name, make, _mk, nout in wl["ops"]:
        st = engine.Stats()
        assert engine.process(make(), outs[:nout], [src], engine.Options(Device=local_rank, Stats=st)) is None
        torch.cuda.synchronize()
        print(json.dumps({"op": name, "cells": st.Cells, "ideal": st.Ideal, "kernel_read": st.KernelRead,
                          "kernel_written": st.KernelWritten, "bands": st.Bands}), flush=True)


def _summary(line, keys):
    return {k: line[k] for k in keys if k in line}


def run_default(args, rank, world, local_rank):
    """The headline workload (the terrain set on 16384 x 16384) and, on one
    GPU, the other configurations' own figures beside it: the focal set on
    8192 x 8192 (per op, roofline and parity), the batched form (512
    rasters, batched over plain) and the served form (40000 x 40000
    mosaic, served over plain, p50 / p99 latency)."""
    import copy

    line = run_ours(args, rank, world, local_rank)
    if world == 1 and not args.no_extra and args.workload == "terrain16k" and not args.side and not args.ops:
        sub = copy.copy(args)
        sub.no_cpu = True
        sub.workload = "focal8k"
        f = run_ours(sub, rank, world, local_rank)
        line["focal8k"] = _summary(f, ["config", "value", "unit", "ms_per_step", "roofline", "per_op", "parity", "e2e"])
        sub.workload = "batch512"
        b = run_batch(sub, rank, world, local_rank)
        line["batch512"] = _summary(b, ["config", "value", "unit", "ms_per_step", "plain_launches",
                                        "batched_over_plain", "roofline", "parity"])
        sub.workload = "serve40k"
        v = run_serve(sub, rank, world, local_rank)
        line["serve40k"] = _summary(v, ["config", "value", "unit", "latency_ms", "plain_launches",
                                        "served_over_plain", "server"])
        sub.workload = "raw8k"
        sub.side = None
        line["raw8k"] = run_raw(sub, rank, world, local_rank)
    return line


def run_reference(args):
    """The reference's CPU implementation of the path, timed on the host:
    the reference (Go) cannot be built here, so this is its restatement,
    the AVX2 lanes of internal/stencil/simd_amd64.go (radius-1 stencils;
    the scalar kernels for the rest) in the reference's engine structure
    (bands of 2^16 cells, word-level validity), on every host thread, over
    the whole workload each step. It loads the oracle only."""
    wl = workload(args.workload, args.side, args.ops)
    threads = os.cpu_count() or 1
    src = _band(wl, 0, wl["height"])
    for _ in range(args.warmup):
        cpu_run(wl, src, threads, True)
    cells, secs = cpu_run(wl, src, threads, True, args.steps)
    value = cells / secs / 1e6
    line = {
        "impl": "reference", "metric": "Mcells/s (output cells of every op in the set per second)",
        "value": round(value, 1), "unit": "Mcells/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(secs / args.steps * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl["name"], "width": wl["width"], "height": wl["height"], "cell_size": wl["cell_size"],
                   "ops": [o[0] for o in wl["ops"]], "mask": wl["mask"]},
        "cpu_baseline": {"value": round(value, 1), "unit": "Mcells/s", "cores": threads, "kind": "restated-avx2",
                         "sample": f"the whole workload ({wl['width']}x{wl['height']}, every op) per step; AVX2 lanes "
                                   f"after internal/stencil/simd_amd64.go, scalar kernels elsewhere"},
        "e2e": {"value": round(value, 1), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="terrain16k",
                    choices=["terrain16k", "slope2k", "slope8k", "pipeline8k", "focal8k", "batch512", "serve40k",
                             "raw8k"])
    ap.add_argument("--tune-cache", action="store_true", help="keep the batch autotuner's choices in a file")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="the headline workload alone (no focal, batched and served figures beside it)")
    ap.add_argument("--side", type=int, default=None, help="raster side override (profiling captures)")
    ap.add_argument("--band", type=int, default=None, help="serving: rows per unit of the radius-1 batch kernels")
    ap.add_argument("--ops", default=None, help="comma-separated ops of the workload to keep (profiling captures)")
    ap.add_argument("--stats", action="store_true",
                    help="print each op's engine.Stats from one plain call (for an ncu DRAM-bytes capture) and exit")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if args.stats:
        run_stats(args, local_rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.workload == "batch512":
            line = run_batch(args, rank, world, local_rank)
        elif args.workload == "serve40k":
            line = run_serve(args, rank, world, local_rank)
        elif args.workload == "raw8k":
            line = run_raw(args, rank, world, local_rank)
        else:
            line = run_default(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
