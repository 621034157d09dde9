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
(focal ops on 8192 x 8192, r = 1..8).

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

def terrain_ops(cell_size):
    from strata_b200 import terrain, transfer

    o = dict(CellSize=cell_size)
    return [
        ("gradient", lambda: terrain.gradient_stage(terrain.GradientOptions(**o)), 2),
        ("slope", lambda: terrain.slope_stage(terrain.SlopeOptions(**o)), 1),
        ("aspect", lambda: terrain.aspect_stage(terrain.AspectOptions(**o)), 1),
        ("hillshade", lambda: terrain.hillshade_stage(terrain.HillshadeOptions(Azimuth=315, Altitude=45,
                                                                               ZFactor=1, **o)), 1),
        ("curvature_profile", lambda: terrain.curvature_stage(terrain.CurvatureOptions(Type=0, **o)), 1),
        ("curvature_plan", lambda: terrain.curvature_stage(terrain.CurvatureOptions(Type=1, **o)), 1),
        ("curvature_mean", lambda: terrain.curvature_stage(terrain.CurvatureOptions(Type=2, **o)), 1),
        ("tri", lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=0, Radius=1)), 1),
        ("tpi", lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=2, Radius=1)), 1),
        ("roughness", lambda: terrain.ruggedness_stage(terrain.RuggednessOptions(Type=3, Radius=1)), 1),
        ("slope_lookup_reclass", lambda: terrain.slope_stage(terrain.SlopeOptions(**o))
         .extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS)).extend(transfer.reclass_stage(BREAKS, VALUES)), 1),
    ]


def focal_ops():
    from strata_b200 import engine, focal, synth

    ops = []
    for r in range(1, 9):
        w = synth.uniform_weights((2 * r + 1) ** 2, 0x5EED0003 + r)
        ops.append((f"correlate_r{r}", lambda w=w, r=r: focal.weights_stage(focal.WeightsOptions(r, w), False), 1))
    g = focal.Gaussian(8, 2.5)
    ops.append(("gaussian_r8", lambda: focal.separable_stage(focal.SeparableOptions(8, g, g)), 1))
    for r in (3, 8):
        for name, op in (("mean", engine._lib.OP_MEAN), ("min", engine._lib.OP_MIN), ("max", engine._lib.OP_MAX)):
            ops.append((f"{name}_r{r}", lambda r=r, op=op: focal.box_stage(focal.BoxOptions(r), op), 1))
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
    from strata_b200 import synth

    if name == "terrain16k":
        n, seed, cs = side or 16384, 0x5EED0002, 10
        cells = synth.fbm_dem(n, n, seed)
        valid = synth.block_mask(n, n, seed, 0.02)
        return dict(name=f"terrain set on {n}x{n} f32 DEM", width=n, height=n, cells=cells, valid=valid,
                    ops=terrain_ops(cs), cell_size=cs, mask="2% NoData in 8x8 blocks")
    if name == "slope2k":
        n, seed, cs = side or 2048, 0x5EED0001, 30
        from strata_b200 import terrain

        return dict(name=f"Slope on {n}x{n} f32 DEM", width=n, height=n, cells=synth.fbm_dem(n, n, seed),
                    valid=synth.block_mask(n, n, seed, 0.02), cell_size=cs, mask="2% NoData in 8x8 blocks",
                    ops=[("slope", lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=cs)), 1)])
    if name == "slope8k":
        n, seed, cs = side or 8192, 0x5EED0001, 30
        from strata_b200 import terrain

        return dict(name=f"Slope on {n}x{n} f32 DEM", width=n, height=n, cells=synth.fbm_dem(n, n, seed),
                    valid=synth.block_mask(n, n, seed, 0.02), cell_size=cs, mask="2% NoData in 8x8 blocks",
                    ops=[("slope", lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=cs)), 1)])
    if name == "pipeline8k":
        n, seed, cs = side or 8192, 0x5EED0002, 10
        from strata_b200 import terrain, transfer

        return dict(name=f"Slope->Lookup->Reclass on {n}x{n} f32 DEM", width=n, height=n,
                    cells=synth.fbm_dem(n, n, seed), valid=synth.block_mask(n, n, seed, 0.02), cell_size=cs,
                    mask="2% NoData in 8x8 blocks",
                    ops=[("slope_lookup_reclass", lambda: terrain.slope_stage(terrain.SlopeOptions(CellSize=cs))
                          .extend(transfer.lookup_stage(SLOPE_XS, SLOPE_YS))
                          .extend(transfer.reclass_stage(BREAKS, VALUES)), 1)])
    if name == "focal8k":
        n, seed = side or 8192, 0x5EED0003
        return dict(name=f"focal ops on {n}x{n} f32 raster", width=n, height=n, cells=synth.normal_trend(n, n, seed),
                    valid=synth.cell_mask(n, n, seed, 0.05), ops=focal_ops(), cell_size=None,
                    mask="5% random NoData cells")
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
# The CPU leg: the oracle on a row band.

def cpu_run(wl, rows, nthreads, reps=1):
    """Runs every op of the workload with the oracle over the first `rows`
    rows of the input; returns (cells processed, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import host_raster, like, run_oracle

    src = host_raster(np.ascontiguousarray(wl["cells"][:rows]), wl["valid"][:rows])
    outs = [like(src), like(src)]
    total, t0 = 0, time.perf_counter()
    for _ in range(reps):
        for _name, mk, nout in wl["ops"]:
            run_oracle(mk(), src, outs[:nout], nthreads=nthreads)
            total += src.width * src.height
    return total, time.perf_counter() - t0


def cpu_baseline(wl, target_s=10.0):
    threads = os.cpu_count() or 1
    rows = min(wl["height"], max(64, (1 << 22) // wl["width"]))
    cells, secs = cpu_run(wl, rows, threads)
    reps = max(1, int(target_s / max(secs, 1e-3)))
    cells, secs = cpu_run(wl, rows, threads, reps)
    return {"value": cells / secs / 1e6, "unit": "Mcells/s", "cores": threads, "kind": "port",
            "sample": f"{rows} rows x {wl['width']} cells, every op of the set, {reps} pass(es), {secs:.1f} s"}


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
    ops = [(name, mk(), nout) for name, mk, nout in wl["ops"]]

    def step(events=None):
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
    torch.cuda.synchronize()

    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()

    per_op = [[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] for _ in ops]
    op_ms = [0.0] * len(ops)
    # Per-op durations, from a separate pass of K steps with events between ops.
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            step(per_op)
            torch.cuda.synchronize()
            for i in range(len(ops)):
                op_ms[i] += per_op[i][0].elapsed_time(per_op[i][1]) / args.steps

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
    top = max(range(len(ops)), key=lambda i: op_ms[i])
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(args.workload, {}).get(ops[top][0])
        except Exception:
            traffic = None
    top_bytes = alg_bytes(n, ops[top][2], masked)
    achieved = top_bytes / (op_ms[top] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": ops[top][0], "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "alg_bytes_per_launch": int(top_bytes)}

    # e2e: the public API with host (page-locked) buffers, every copy inside
    # the timed region: one process_features call (terrain.Features) for
    # every op of the set, the pipeline included, so the DEM crosses once
    # and each output's copy back overlaps the next op's kernels.
    host_src = Float32Raster(host_cells.numpy(), W, H, W, host_mask.numpy().view(np.uint64), 0)
    n_outs = sum(nout for _n, _s, nout in ops)
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

    launches_per_step = sum(1 + (nout if masked else 0) for _n, _s, nout in ops)
    line = {
        "metric": "Mcells/s (output cells of every op in the set per second)", "value": round(value, 1),
        "unit": "Mcells/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl["name"], "width": W, "height": H, "cell_size": wl["cell_size"],
                   "ops": [o[0] for o in ops], "mask": wl["mask"], "l2": "inputs larger than L2 (no flush)",
                   "parallelism": f"independent rasters x{world}"},
        "roofline": roofline, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(), "per_op": per,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl)
    if rank == 0:
        print(json.dumps(line), flush=True)


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
    }
    b.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


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
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args):
    wl = workload(args.workload, args.side, args.ops)
    threads = os.cpu_count() or 1
    rows = min(wl["height"], max(64, (1 << 22) // wl["width"]))
    for _ in range(args.warmup):
        cpu_run(wl, rows, threads)
    cells, secs = 0, 0.0
    for _ in range(args.steps):
        c, s = cpu_run(wl, rows, threads)
        cells += c
        secs += s
    value = cells / secs / 1e6
    line = {
        "impl": "reference", "metric": "Mcells/s (output cells of every op in the set per second)",
        "value": round(value, 1), "unit": "Mcells/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(secs / args.steps * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl["name"], "width": wl["width"], "height": wl["height"],
                   "ops": [o[0] for o in wl["ops"]], "mask": wl["mask"]},
        "cpu_baseline": {"value": round(value, 1), "unit": "Mcells/s", "cores": threads, "kind": "port",
                         "sample": f"{rows} rows x {wl['width']} cells of the workload, every op, per step"},
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
                    choices=["terrain16k", "slope2k", "slope8k", "pipeline8k", "focal8k", "batch512", "serve40k"])
    ap.add_argument("--tune-cache", action="store_true", help="keep the batch autotuner's choices in a file")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--side", type=int, default=None, help="raster side override (profiling captures)")
    ap.add_argument("--band", type=int, default=None, help="serving: rows per unit of the radius-1 batch kernels")
    ap.add_argument("--ops", default=None, help="comma-separated ops of the workload to keep (profiling captures)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.workload == "batch512":
            run_batch(args, rank, world, local_rank)
        elif args.workload == "serve40k":
            run_serve(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
