"""Benchmark: Mcells/s of the plain GPU path on the synthetic 4097 x 4097 terrain at 0.5 m
(8-octave fBm source, 200,000 craters, 1,000,000 boulders of which those resolved are drawn).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tgb200|reference]

A step evaluates one whole tile: the source fill, the crater layer and the boulder layer.
`value` is device-resident throughput (inputs already in HBM); `e2e` runs the same step through
the public C ABI with host buffers (tg_evaluate: layer inputs copied in from pinned memory, heights
copied out, every step). With N ranks (torchrun) each rank evaluates its own tile, with no
exchange (weak scaling). `--impl reference` times the reference CPU path on a bounded window of
the same terrain with every host core. Rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mcells/s at <=1e-3 m err: served/batched vs plain GPU; p50/p99 tile ms"
UNIT = "Mcells/s"
SIDE = 4097
PIXEL = 0.5
# Counted from terraingen_b200/csrc/noise_math.cuh (perlin_fbm2), per cell and octave: octave
# key hash and offsets 21, turn 6, lattice 4, split 6, 4 corner hashes 45, 4 gradients 56 plus 2
# offsets, 2 fades 14, lerps and scale 10, sums 5, turn update 6, loop 3.
NOISE_OPS_PER_CELL_OCTAVE = 180
# Counted from terraingen_b200/csrc/crater_math.cuh (fast_contribution) per (cell, crater) pair of
# a Fassett-Thomson crater with 11 outline harmonics: distance and radii 12, outline share 14,
# direction 18, first-harmonic rotation and kept share 14, 11 harmonics x 10, scale and division
# 10, profile 18, resolution and FP64 sum 4.
CRATER_OPS_PER_PAIR = 200
# Counted from terraingen_b200/csrc/boulders.cu per (cell, boulder) pair: window test 6, offset
# and hypot 12, dome band average (2 sqrt, 2 asin, clamps) 60, max-composite 4; FP64.
BOULDER_OPS_PER_PAIR = 82
# DRAM bytes per launch from the ncu capture of this workload (profiles/terrain4097_kernels.md).
TRAFFIC = {"noise": 0.062e6 + 10.28e6, "craters": 136.5e6 + 27.0e6, "boulders": 61.9e6 + 7.9e6}
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tgb200", choices=["tgb200", "reference"])
    p.add_argument("--cpu-window", type=int, default=1025,
                   help="side of the window the CPU baseline evaluates")
    return p.parse_args()


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(steps, warmup, window, quiet=False):
    """The reference CPU path on a `window`^2 window of the terrain, every host core: (Mcells/s,
    seconds per evaluation, evaluations timed)."""
    from oracle import harness as H
    from terraingen_b200.workloads import terrain4097_reference_scene

    lib = H.reference()
    grid, fr, craters, boulders = terrain4097_reference_scene(window, PIXEL)
    scene = H.make_scene(grid, source_fractals=fr, craters=craters, boulders=boulders)
    for _ in range(warmup):
        H.evaluate(lib, scene, 0, 0)
    times = []
    deadline = time.perf_counter() + 30.0
    for i in range(max(steps, 1)):
        _, ms = H.evaluate(lib, scene, 0, 0)
        times.append(ms * 1e-3)
        if time.perf_counter() > deadline and i >= 0:
            break
    per = float(np.median(times))
    return grid.cells / per / 1e6, per, len(times), grid


def run_reference(args, rank, world):
    if rank != 0:
        return
    value, per, n, grid = cpu_sample(args.steps, args.warmup, args.cpu_window)
    cores = os.cpu_count()
    sample = (f"{grid.width}x{grid.height} window at {PIXEL} m of the 4097^2 terrain (same fBm, "
              f"crater and boulder densities), reference CPU path, {n} evaluations")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
        "n_gpus": args.gpus, "steps": n, "warmup": args.warmup, "ms_per_step": round(per * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": "terrain4097 window", "cells": grid.cells, "pixel_m": PIXEL},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def scan_launches(n):
    """Kernel launches of one exclusive scan of n counts (craters.cu launch_exclusive_scan)."""
    blocks = (n + 1 + 1023) // 1024
    return 1 if blocks == 1 else 2 + scan_launches(blocks)


def main():
    args = parse()
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch

    from terraingen_b200 import Device
    from terraingen_b200.build import build
    from terraingen_b200.workloads import terrain4097

    if rank == 0:
        build()
    barrier(world)
    torch.cuda.set_device(local)
    dev = Device(local)
    # Each rank's own tile, side by side along x (independent tiles, no exchange).
    w = terrain4097(SIDE, PIXEL, cx=rank * SIDE * PIXEL)
    stream = torch.cuda.current_stream()
    rec = torch.from_numpy(w.crater_records.view(np.uint8)).cuda()
    data = torch.from_numpy(w.crater_data).cuda()
    foot = torch.from_numpy(w.crater_footprints).cuda()
    bould = torch.from_numpy(w.boulders).cuda()
    heights = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step(timers=None):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if timers is not None \
            else None
        if ev:
            ev[0].record(stream)
        dev.noise_source(w.fractals, w.grid, heights, w.elevation)
        if ev:
            ev[1].record(stream)
        dev.craters_apply(w.crater_kernel, rec, data, w.grid, heights, footprints=foot)
        if ev:
            ev[2].record(stream)
        dev.boulders_bake(bould, w.grid, heights, width=w.boulder_width)
        if ev:
            ev[3].record(stream)
            timers.append(ev)

    for _ in range(args.warmup):
        flush.fill_(1.0)
        step()
    torch.cuda.synchronize()
    alu_peak = dev.measure_alu()
    barrier(world)
    torch.cuda.synchronize()
    timers = []
    with Clocks(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)  # outside the timed events: the L2 holds nothing of the last step
            step(timers)
        torch.cuda.synchronize()
    barrier(world)
    counters = dev.counters()
    phases = np.array([[e[i].elapsed_time(e[i + 1]) for i in range(3)] for e in timers])
    step_ms = float(phases.sum(axis=1).mean())
    total_s = max_over_ranks(float(phases.sum()) * 1e-3, world)
    value = world * w.cells * args.steps / total_s / 1e6

    # End to end through the public C ABI with host buffers from pinned memory.
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_rec, h_data, h_foot, h_b = (pin(w.crater_records.view(np.uint8)), pin(w.crater_data),
                                  pin(w.crater_footprints), pin(w.boulders))
    h_heights = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32).pin_memory()
    h_out = h_heights.numpy()

    def e2e_step():
        dev.evaluate(w.grid, h_out, fractals=w.fractals, elevation=w.elevation,
                     craters=(w.crater_kernel, h_rec.view(w.crater_records.dtype), h_data,
                              h_foot),
                     boulders=h_b, boulder_width=w.boulder_width)

    for _ in range(args.warmup):
        e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * w.cells * args.steps / e2e_s / 1e6
    h2d = w.input_bytes()
    d2h = w.cells * 4

    # Parity of the device-resident and end-to-end results (same inputs, same bits).
    same = bool(torch.equal(heights.cpu(), h_heights))

    if rank != 0:
        return
    noise_ms = float(phases[:, 0].mean())
    crater_ms = float(phases[:, 1].mean())
    boulder_ms = float(phases[:, 2].mean())
    octaves = int(w.fractals[0]["octaves"])
    work = {"noise": (w.cells * octaves * NOISE_OPS_PER_CELL_OCTAVE, noise_ms,
                      "fbm_kernel (fBm source)", f"{NOISE_OPS_PER_CELL_OCTAVE} per cell-octave"),
            "craters": (counters["crater_pairs"] * CRATER_OPS_PER_PAIR, crater_ms,
                        "crater pipeline (count, scan, scatter, crater_shape_kernel)",
                        f"{CRATER_OPS_PER_PAIR} per (cell, crater) pair, "
                        f"{counters['crater_pairs']} pairs"),
            "boulders": (counters["boulder_pairs"] * BOULDER_OPS_PER_PAIR, boulder_ms,
                         "boulder pipeline (count, scan, scatter, boulder_bake_kernel)",
                         f"{BOULDER_OPS_PER_PAIR} per (cell, boulder) pair, "
                         f"{counters['boulder_pairs']} pairs")}
    dominant = max(work, key=lambda k: work[k][1])
    ops, ms, kernel_name, unit_note = work[dominant]
    achieved = ops / (ms * 1e-3) / 1e12
    peak = alu_peak / 1e12
    nbins = ((w.grid.width + 31) // 32) * ((w.grid.height + 31) // 32)
    launches = 1 + (3 + scan_launches(nbins)) * 2  # noise; count, scan, scatter, shape/bake x 2
    cpu_value, cpu_per, cpu_n, cpu_grid = cpu_sample(1, 1, args.cpu_window)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded): fBm source, reference-exact crater batch, stand-in boulders",
        "config": {"workload": "terrain4097: 4097x4097 at 0.5 m, 8-octave fBm + 200k craters + "
                               "1M boulders (resolved ones drawn)",
                   "cells_per_gpu": w.cells, "craters_on_tile": int(len(w.crater_records)),
                   "boulders_drawn": int(len(w.boulders)), "l2": "flushed between steps",
                   "parallelism": f"replicas x{world} (one tile per GPU)"},
        "phases_ms": {"noise": round(noise_ms, 4), "craters": round(crater_ms, 4),
                      "boulders": round(boulder_ms, 4)},
        "roofline": {"kernel": kernel_name, "bound": "alu",
                     "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "Tops/s",
                     "frac": round(achieved / peak, 3) if peak else None,
                     "peak_source": "measured IMAD+FFMA lane-op rate (tg_measure_alu) on this GPU",
                     "algorithmic_ops": unit_note, "traffic": TRAFFIC[dominant],
                     "traffic_source": "ncu dram__bytes_read+write of the shaping/bake/fill "
                                       "kernel, profiles/terrain4097_kernels.md",
                     "others": {k: {"ms": round(v[1], 4),
                                    "achieved": round(v[0] / (v[1] * 1e-3) / 1e12, 3)}
                                for k, v in work.items() if k != dominant}},
        "cpu_baseline": {"value": round(cpu_value, 3), "unit": UNIT, "cores": os.cpu_count(),
                         "kind": "reference",
                         "sample": f"{cpu_grid.width}x{cpu_grid.height} window of the same terrain "
                                   f"on the reference CPU path, {cpu_per * 1e3:.0f} ms"},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "matches_device_path": same},
        "gpu_launches": int(launches * args.steps),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
