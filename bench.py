"""Benchmark: Mcells/s of the plain GPU path on the synthetic 4097 x 4097 terrain at 0.5 m
(8-octave fBm source; 200,000 craters with 5 % central peaks and terraced rims above 200 m, as
terraingen_b200.workloads maps them onto the reference's options; 1,000,000 boulders of which
those resolved are drawn), and under "forms" the batched form on 4096 uneven tiles, the served
form on a camera request stream and the DEM refinement, each against the plain per-tile path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tgb200|reference]

A step evaluates one whole tile: the source fill, the crater layer and the boulder layer.
`value` is device-resident throughput (layer inputs already in HBM). `e2e` starts each step from
the layers' definitions through the public C ABI: the crater batch (population, terraces and
peaks on the host threads, apply order and records on the device: tg_crater_batch_device, its
plan copied in from pinned memory), the boulders placed on the host and copied in, the tile
evaluated (tg_evaluate) and its heights copied out to pinned memory; `e2e.host_records` is the
same with the batch made on the host (tg_crater_batch) and every input passed as host buffers
(inputs copied in, heights copied out inside tg_evaluate). `dropin` times the
reference's own Terrain::Evaluate with Backend::Cuda on this library against Backend::Cpu. With N
ranks each rank evaluates its own tile, with no exchange (weak scaling); `--gpus N` without
torchrun starts the N ranks itself. `--impl reference` times the reference CPU path on a bounded
window of the same terrain with every host core. Rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from terraingen_b200 import ranks  # noqa: E402

METRIC = "Mcells/s at <=1e-3 m err: served/batched vs plain GPU; p50/p99 tile ms"
UNIT = "Mcells/s"
SIDE = 4097
PIXEL = 0.5
# Counted from terraingen_b200/csrc/noise_math.cuh (perlin_fbm2), per cell and octave: octave
# key hash and offsets 21, turn 6, lattice 4, split 6, 4 corner hashes 45, 4 gradients 56 plus 2
# offsets, 2 fades 14, lerps and scale 10, sums 5, turn update 6, loop 3.
NOISE_OPS_PER_CELL_OCTAVE = 180
# Counted from the reference's crater kernel (include/terraingen/layers/kernels/craters.h:
# KernelProfileDistance, ComplexProfileHeight / FassettThomsonShape, ApplyCraterKernel) per
# (cell, crater) pair of the synthetic terrain's craters (11 outline harmonics; a transcendental
# counts one): offset and distance 6, outline share 7, angle 1, 11 harmonics x 7 (k theta, phase,
# cos, amplitude, kept share's pow, product, sum) 77, scale and division 2, reach test 1, profile
# 8, resolution and the add 2: 104, plus the ellipse of 5 % of craters (10): 105.
CRATER_OPS_PER_PAIR = 105
# Thread instructions the lean crater kernel executes per pair, measured with ncu on this
# workload (smsp__inst_executed x active lanes / pairs: 771.3 M x 29.79 / 64,216,893): the
# issue-rate view of the same work (loads, the queue, compares and selects).
CRATER_THREAD_INST_PER_PAIR = 358
# Counted from terraingen_b200/csrc/boulders.cu per (cell, boulder) pair: window test 6, offset
# and hypot 12, dome band average (2 sqrt, 2 asin, clamps) 60, max-composite 4; FP64.
BOULDER_OPS_PER_PAIR = 82
# DRAM bytes (read + write) per launch from the ncu captures of this workload: the fBm kernel,
# the lean crater shaping kernel (as built now: 113.3 + 25.9 MB) and the boulder bake.
TRAFFIC = {"noise": 0.062e6 + 10.28e6, "craters": 113.33e6 + 25.86e6, "boulders": 61.9e6 + 7.9e6}
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tgb200", choices=["tgb200", "reference"])
    p.add_argument("--cpu-window", type=int, default=1025,
                   help="side of the window the CPU baseline evaluates")
    p.add_argument("--tiles", type=int, default=4096,
                   help="tiles of the batched form's uneven-tile workload (0 skips it)")
    p.add_argument("--variant", type=int, default=-1,
                   help="batched kernel shape (tg_batch_variant index); -1 runs the autotuner")
    p.add_argument("--batched-only", action="store_true",
                   help="run the batched form alone and print its line (profiling)")
    p.add_argument("--serve-seconds", type=float, default=3.0,
                   help="length of the real-time request stream of the served form (0 skips it)")
    p.add_argument("--dem-steps", type=int, default=5,
                   help="timed steps of the DEM refinement form (0 skips it)")
    p.add_argument("--dem-side", type=int, default=20481,
                   help="output side of the DEM refinement form (20481; smaller for profiling)")
    p.add_argument("--served-only", action="store_true",
                   help="run the served form alone and print its line (profiling)")
    p.add_argument("--dem-only", action="store_true",
                   help="run the DEM refinement form alone and print its line (profiling)")
    return p.parse_args()


def dist_setup(n):
    r = ranks.setup("nccl")
    return r.rank, r.world, r.local


def _ranks(world):
    return ranks.Ranks(int(os.environ.get("RANK", "0")), world,
                       int(os.environ.get("LOCAL_RANK", "0")), "cuda")


def barrier(world):
    ranks.barrier(_ranks(world))


def max_over_ranks(value, world):
    return ranks.max_over_ranks(value, _ranks(world))


class Clocks:
    """SM clock and throttle reasons sampled every few milliseconds during the timed region, by
    NVML queries (read-only) from a background thread; nvidia-smi when NVML is unavailable."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.max_mhz = None
        self._stop = None
        self._thread = None

    def _handle(self, nv):
        try:
            import torch

            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            handle = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(handle, nv.NVML_CLOCK_SM))
        except Exception:
            return self
        self._stop = threading.Event()

        def poll():
            while not self._stop.is_set():
                try:
                    mhz = nv.nvmlDeviceGetClockInfo(handle, nv.NVML_CLOCK_SM)
                    reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(handle)
                    self.samples.append((float(mhz), int(reasons)))
                except Exception:
                    break
                self._stop.wait(0.002)

        self._thread = threading.Thread(target=poll, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self):
        import pynvml as nv

        reasons = set()
        for _, bits in self.samples:
            for name, const in self.REASONS.items():
                if bits & getattr(nv, const, 0):
                    reasons.add(name)
        sm = [m for m, _ in self.samples]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "NVML, 2 ms"}


FP64_FIXTURE = ROOT / "tests" / "golden" / "fp64.npz"


def fp64_error(got, case, rows=None, cols=None):
    """Max and RMS height error (m) of `got` (the cells of fixture case `case`'s grid, or a
    larger array and the rows / cols slices of the case's window in it) against the FP64 oracle
    heights in tests/golden/fp64.npz (tests/golden/fp64_cases.py)."""
    want = np.load(FP64_FIXTURE)[f"{case}_fp64"]
    got = np.asarray(got)
    if rows is not None:
        got = got[rows, cols]
    err = np.abs(got.reshape(want.shape).astype(np.float64) - want)
    return {"max_err_m": float(err.max()), "rms_err_m": float(np.sqrt(np.mean(err ** 2))),
            "cells": int(want.size)}


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
        "n_gpus": world, "steps": n, "warmup": args.warmup, "ms_per_step": round(per * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"terrain4097 window ({grid.width}x{grid.height} at the tile's "
                               "center): the same stack as the GPU arm's terrain4097 (fBm, 200k "
                               "craters per tile with the peak and terrace mapping, 1M boulders "
                               "per tile)", "cells": grid.cells, "pixel_m": PIXEL},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def scan_launches(n):
    """Kernel launches of one exclusive scan of n counts (craters.cu launch_exclusive_scan)."""
    blocks = (n + 1 + 1023) // 1024
    return 1 if blocks == 1 else 2 + scan_launches(blocks)


def batched_form(dev, args, rank, world, alu_peak):
    """The batched form on uneven tiles (tiles4096): every rank its own 4096 tiles, evaluated in
    one persistent launch replayed from CUDA graphs, against the plain per-tile path on the same
    tiles (tg_noise_source, tg_craters_apply, tg_boulders_bake per tile, device-resident)."""
    import torch

    from terraingen_b200.batch import Batch
    from terraingen_b200.workloads import uneven_tiles

    ts = uneven_tiles(args.tiles, seed=ranks.tiles_seed(rank))
    batch = Batch(dev)
    batch.load(ts)
    out = torch.empty(ts.output_floats, dtype=torch.float32, device="cuda")
    if args.variant >= 0:
        batch.set_variant(args.variant)
        tune_ms = []
    else:
        tune_ms = batch.tune(trials=2)
    for _ in range(args.warmup):
        batch.evaluate(out)
    barrier(world)
    bins, evals, graphs = [], [], []
    with Clocks(torch.cuda.current_device()) as clocks:
        for _ in range(args.steps):
            batch.evaluate(out)  # writes 4 B x cells (far above L2) each step
            st = batch.stats()
            bins.append(st["bin_ms"])
            evals.append(st["evaluate_ms"])
            graphs.append(st["graph_ms"])
    total_s = max_over_ranks(float(np.sum(graphs)) * 1e-3, world)
    value = world * ts.cells * args.steps / total_s / 1e6
    # The fixture's far-out tiles of the set (rank 0's set, 4096 tiles) against the FP64 oracle.
    fp64 = None
    if args.tiles == 4096 and ranks.tiles_seed(rank) == 11:
        host = out.cpu().numpy()
        picks = np.load(FP64_FIXTURE)["tiles_index"]
        worst = []
        for k, i in enumerate(picks):
            g, o, p = ts.grids[i], int(ts.tiles["height_offset"][i]), int(ts.tiles["pitch"][i])
            cells = np.stack([host[o + r * p:o + r * p + g.width] for r in range(g.height)])
            worst.append(fp64_error(cells, f"tile{k}"))
        fp64 = {"tiles": [int(i) for i in picks],
                "max_err_m": max(e["max_err_m"] for e in worst),
                "rms_err_m": float(np.sqrt(np.mean([e["rms_err_m"] ** 2 for e in worst]))),
                "farthest_m": float(max(np.hypot(ts.grids[i].x0, ts.grids[i].y0)
                                        for i in picks))}

    # The plain per-tile path over the same tiles, inputs resident on the device.
    stream = torch.cuda.current_stream()
    per_tile = []
    t = ts.tiles
    for i, g in enumerate(ts.grids):
        r0, rn = int(t["crater_begin"][i]), int(t["crater_count"][i])
        d0 = int(t["data_begin"][i])
        d1 = int(t["data_begin"][i + 1]) if i + 1 < len(ts.grids) else len(ts.crater_data)
        b0, bn = int(t["boulder_begin"][i]), int(t["boulder_count"][i])
        per_tile.append((
            g, rn,
            torch.from_numpy(ts.crater_records[r0:r0 + rn].view(np.uint8).copy()).cuda(),
            torch.from_numpy(ts.crater_data[d0:max(d1, d0 + 1)].copy()).cuda(),
            torch.from_numpy(ts.crater_footprints[3 * r0:3 * (r0 + rn)].copy()).cuda(),
            bn, torch.from_numpy(np.ascontiguousarray(ts.boulders[b0:b0 + bn])).cuda(),
            torch.empty((g.height, g.width), dtype=torch.float32, device="cuda"),
            float(t["boulder_width"][i])))

    def plain():
        for g, rn, rec, dat, foot, bn, bou, h, width in per_tile:
            dev.noise_source(ts.fractals, g, h, ts.elevation)
            if rn:
                dev.craters_apply(ts.crater_kernel, rec, dat, g, h, footprints=foot)
            if bn:
                dev.boulders_bake(bou, g, h, width=width)

    plain()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    plain()
    e1.record(stream)
    torch.cuda.synchronize()
    plain_s = max_over_ranks(e0.elapsed_time(e1) * 1e-3, world)
    plain_value = world * ts.cells / plain_s / 1e6

    # End to end: tg_batch_run from host arrays into pinned host memory (inputs copied in and
    # heights copied out inside each call).
    host_out = torch.empty(ts.output_floats, dtype=torch.float32).pin_memory().numpy()
    batch.run(ts, host_out)
    barrier(world)
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        batch.run(ts, host_out)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = world * ts.cells * e2e_steps / e2e_s / 1e6
    same = bool(np.array_equal(host_out, out.cpu().numpy()))
    st = batch.stats()
    octaves = int(ts.fractals[0]["octaves"])
    eval_ms = float(np.mean(evals))
    ops = (ts.cells * octaves * NOISE_OPS_PER_CELL_OCTAVE + st["crater_pairs"] * CRATER_OPS_PER_PAIR
           + st["boulder_pairs"] * BOULDER_OPS_PER_PAIR)
    achieved = ops / (eval_ms * 1e-3) / 1e12
    peak = alu_peak / 1e12
    batch.close()
    return {
        "workload": f"tiles{args.tiles}: sides log-uniform 65-1025, 0.25-2 m/px, centers within "
                    "1.7e6 m (polar frame of a 1737.4 km sphere); terrain4097 stack at 1/10 "
                    "crater and boulder density",
        "tiles": int(len(ts.tiles)), "cells_per_gpu": ts.cells,
        "craters": int(len(ts.crater_records)), "boulders": int(len(ts.boulders)),
        "value": round(value, 3), "unit": UNIT,
        "ms_per_step": round(float(np.mean(graphs)), 4),
        "bin_ms": round(float(np.mean(bins)), 4), "evaluate_ms": round(eval_ms, 4),
        "plain_per_tile": {"value": round(plain_value, 3), "unit": UNIT,
                           "ms": round(plain_s * 1e3, 3),
                           "path": "tg_noise_source + tg_craters_apply + tg_boulders_bake per tile"},
        "speedup_vs_plain": round(value / plain_value, 2),
        "fp64": fp64,
        "kernel_shape": {"bin": [st["bin_width"], st["bin_height"]],
                         "cells_per_thread": st["cells_per_thread"], "ctas": st["ctas"]},
        "autotuner_ms": [None if not np.isfinite(m) else round(m, 3) for m in tune_ms],
        "graph": {"captures": st["captures"], "replays": st["replays"]},
        "roofline": {"kernel": "batch_evaluate_kernel (persistent: fBm + craters + boulders)",
                     "bound": "alu", "achieved": round(achieved, 3), "peak": round(peak, 3),
                     "unit": "Tops/s", "frac": round(achieved / peak, 3) if peak else None,
                     "algorithmic_ops": f"{NOISE_OPS_PER_CELL_OCTAVE} per cell-octave + "
                                        f"{CRATER_OPS_PER_PAIR} per crater pair "
                                        f"({st['crater_pairs']}) + {BOULDER_OPS_PER_PAIR} per "
                                        f"boulder pair ({st['boulder_pairs']})"},
        "accuracy": "source within 1e-4 m of the FP64 oracle at 1.7e6 m "
                    "(tests/test_batch_gpu.py); craters and boulders evaluate the plain path's "
                    "pairs, within 1e-4 m of it",
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                "h2d_bytes_per_step": int(ts.input_bytes()),
                "d2h_bytes_per_step": int(ts.output_floats * 4), "matches_device_path": same},
        "gpu_launches_per_step": int(6 + 2 * scan_launches(st["bins"]) + 1),
        "clocks": clocks.summary(),
        "l2": "output (4 B per cell) far above L2, written every step",
    }


def dem_form(dev, args, rank, world):
    """The DEM refinement (dem20481): 2x2 patches refined by diamond-square from a 2049^2 DEM at
    5 m to 20481^2 at 0.5 m, chained with Height seams on the device (PatchChain: tg_seam_samples,
    tg_seam_solve, tg_seam_fill per link), then 2,000,000 craters. A step is the whole grid:
    the four refinements, the three seam links and the crater layer, inputs resident."""
    import torch

    from terraingen_b200.chain import PatchChain, Seams
    from terraingen_b200.workloads import dem20481

    w = dem20481(args.dem_side, (args.dem_side - 1) // 10 + 1, seed=ranks.dem_seed(rank))
    pg = w.post_grid
    posts = torch.empty((pg.height, pg.width), dtype=torch.float32, device="cuda")
    dev.noise_source(w.fractals, pg, posts, 0.0)
    patches = [torch.empty((win.height, win.width), dtype=torch.float32, device="cuda")
               for win in w.windows]
    seams = Seams("height", decay_length=w.decay_length, levels=4, sweeps=2, coarsest_sweeps=20)
    chain = PatchChain(dev, w.grid, w.windows, seams)
    rec = torch.from_numpy(w.crater_records.view(np.uint8)).cuda()
    data = torch.from_numpy(w.crater_data).cuda()
    foot = torch.from_numpy(w.crater_footprints).cuda()
    stream = torch.cuda.current_stream()

    def step(timers=None, links=None):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        for k, win in enumerate(w.windows):
            dev.ds_refine(posts, pg, win.grid(w.grid), patches[k], w.fractal_dimension, w.scale,
                          w.seeds[k])
        ev[1].record(stream)
        heights = chain.compose(patches, links)
        ev[2].record(stream)
        dev.craters_apply(w.crater_kernel, rec, data, w.grid, heights, footprints=foot)
        ev[3].record(stream)
        if timers is not None:
            timers.append(ev)
        return heights

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    timers, links = [], []
    with Clocks(torch.cuda.current_device()) as clocks:
        for _ in range(args.dem_steps):
            step(timers, links)  # writes 1.68 GB of heights (far above L2) every step
        torch.cuda.synchronize()
    counters = dev.counters()
    phases = np.array([[e[i].elapsed_time(e[i + 1]) for i in range(3)] for e in timers])
    link_ms = np.array([[[lk[i].elapsed_time(lk[i + 1]) for i in range(3)] for lk in links]])
    total_s = max_over_ranks(float(phases.sum()) * 1e-3, world)
    value = world * w.cells * args.dem_steps / total_s / 1e6
    heights = chain.heights
    finite = bool(torch.isfinite(heights).all())

    # End to end: the DEM posts copied in from pinned memory and the heights copied out to pinned
    # memory every step, around the same device work. Each step's heights are snapshotted on the
    # device and read back on a copy stream while the next step refines, the way a producer of
    # tiles streams them out; the timed region ends when the last step's heights are on the host.
    host_posts = torch.empty((pg.height, pg.width), dtype=torch.float32).pin_memory()
    host_posts.copy_(posts)
    host_out = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32).pin_memory()
    snapshot = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32, device="cuda")
    copier = torch.cuda.Stream()
    barrier(world)
    t0 = time.perf_counter()
    e2e_steps = max(1, args.dem_steps)
    for _ in range(e2e_steps):
        posts.copy_(host_posts, non_blocking=True)
        out = step()
        stream.wait_stream(copier)  # the previous step's read-back is done with the snapshot
        snapshot.copy_(out)
        copier.wait_stream(stream)
        with torch.cuda.stream(copier):
            host_out.copy_(snapshot, non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    same_out = bool(torch.equal(host_out, chain.heights.cpu()))
    accuracy = dem_accuracy(dev)
    e2e_value = world * w.cells * e2e_steps / e2e_s / 1e6
    solves = chain.solves
    per_link = link_ms.reshape(-1, len(w.windows) - 1, 3).mean(axis=0)
    return {
        "workload": f"dem{w.grid.width}: {w.post_grid.width}^2 DEM at 5 m (12-octave fBm, 20 km, "
                    "+-2000 m) refined 10x by "
                    "diamond-square (F 2.2, scale 1.5 m, 4 levels, bilinear) to 20481^2 at 0.5 m "
                    "as 2x2 patches (own seeds, 64-cell overlap) chained with Height seams "
                    "(3 L = 64 cells, 4-level V-cycle, Jacobi smoother, FP64 PCG to 1e-10), then "
                    "2,000,000 craters (D^-2 on [1, 100] m)",
        "cells_per_gpu": w.cells, "craters": int(len(w.crater_records)),
        "value": round(value, 3), "unit": UNIT,
        "ms_per_step": round(float(phases.sum(axis=1).mean()), 3),
        "phases_ms": {"diamond_square": round(float(phases[:, 0].mean()), 3),
                      "seam_chain": round(float(phases[:, 1].mean()), 3),
                      "craters": round(float(phases[:, 2].mean()), 3)},
        "seam_links": [{"samples_ms": round(float(a), 3), "seam_solve_call_ms": round(float(b), 3),
                        "fill_ms": round(float(c), 3),
                        **{("pcg_ms" if k == "solve_ms" else k):
                           (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()}}
                       for (a, b, c), st in zip(per_link, solves)],
        "crater_pairs": int(counters["crater_pairs"]),
        "fp64": accuracy,
        "all_cells_filled": finite,
        "accuracy": "diamond-square within 1e-3 m of the reference (tests/test_ds_gpu.py); seam "
                    "fields within 1e-4 m of the reference's converged PCG, Feather and the gap "
                    "fill bit-exact (tests/test_seams_gpu.py); craters as the plain path",
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT,
                "h2d_bytes_per_step": int(pg.cells * 4),
                "d2h_bytes_per_step": int(w.cells * 4), "matches_device_path": same_out,
                "overlap": "each step's heights read back on a copy stream during the next step"},
        "clocks": clocks.summary(),
        "l2": "output (1.68 GB) far above L2, written every step",
    }


def next_rows_form(dev):
    """The stages beyond the per-cell path, timed once each: the dem20481 crater population drawn
    on the device against the host restatement, a synthetic source on a sphere, and a GeoTIFF of
    a 4097^2 grid written from device memory."""
    import math
    import os
    import tempfile

    import torch

    from terraingen_b200 import GridSpec
    from terraingen_b200.layouts import fractal
    from terraingen_b200.workloads import (crater_population, generate_craters,
                                           generate_craters_device)

    side = 20481 * 0.5
    pop = crater_population(11, 2.0e6 / (side * side * (1.0 - 100.0 ** -2)), 1.0, 100.0)
    region = (0.0, 0.0, side, side)
    t0 = time.perf_counter()
    host = generate_craters(pop, region)
    host_s = time.perf_counter() - t0
    generate_craters_device(dev, pop, region)
    t0 = time.perf_counter()
    drawn = generate_craters_device(dev, pop, region)
    device_s = time.perf_counter() - t0
    radius = 1737400.0
    g = GridSpec(4097, 4097, 10.0, 1.0, 0.5 / (radius * math.pi / 180.0))
    fr = np.array([fractal(seed=1, wavelength=512.0, amplitude=5.0, octaves=8)])
    body = torch.empty((4097, 4097), dtype=torch.float32, device="cuda")
    dev.noise_source_body(fr, g, radius, body)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        dev.noise_source_body(fr, g, radius, body)
    e1.record()
    torch.cuda.synchronize()
    body_ms = e0.elapsed_time(e1) / 5
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "dem.tif")
        grid = (4097, 4097, (0.0, 0.5, 0.0, 0.0, 0.0, -0.5))
        dev.geotiff_write(path, [body], grid, nodata=float("nan"))
        t0 = time.perf_counter()
        dev.geotiff_write(path, [body], grid, nodata=float("nan"))
        tiff_s = time.perf_counter() - t0
        tiff_bytes = os.path.getsize(path)
    return {
        "crater_population": {"craters": int(len(drawn["x"])), "device_ms": round(device_s * 1e3, 2),
                              "host_ms": round(host_s * 1e3, 1),
                              "ids_match_host": bool(np.array_equal(drawn["id"], host["id"])),
                              "identical_to_host": bool(all(
                                  np.array_equal(drawn[k], host[k])
                                  for k in ("x", "y", "diameter", "age", "id")))},
        "body_source": {"cells": 4097 * 4097, "ms": round(body_ms, 3),
                        "mcells_per_s": round(4097 * 4097 / body_ms / 1e3, 1),
                        "stack": "one 8-octave Perlin fBm on a sphere of 1737.4 km"},
        "geotiff_lzw": {"cells": 4097 * 4097, "seconds": round(tiff_s, 3), "bytes": int(tiff_bytes),
                        "from": "device memory, 256-pixel LZW tiles, file write included"},
    }


def served_form(dev, args, rank, world):
    """The served form on the camera request stream (terraingen_b200/serve.py): the DEM
    refinement's stack (the 12-octave fBm at 5 m posts, refined by diamond-square to each
    request's spacing, craters on top) served by continuous batching, results in device buffers.
    Latency per class at 2000 requests/s in real time; sustained throughput with the stream
    submitted at once; the plain per-request path (per tile: tg_noise_source on its post window,
    tg_ds_refine_window, tg_craters_apply; inputs resident) on tile requests of the same
    stream."""
    import torch

    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import (POST_SPACING, Server, camera_stream, dem_stack_options,
                                       post_lattice, refine_options, run_stream)
    from terraingen_b200.workloads import crater_batch

    opts = dem_stack_options(slots=3, max_batch_cells=8 << 20)
    seconds = max(1.0, min(3.0, args.serve_seconds))
    with Server(dev, opts) as server:
        warm, real, sat = ranks.stream_seeds(rank)
        run_stream(server, camera_stream(0.5, seed=warm), realtime=False, device=True)
        nominal = run_stream(server, camera_stream(seconds, seed=real), realtime=True,
                             device=True)
        sat_reqs = camera_stream(1.0, seed=sat)
        run_stream(server, sat_reqs, realtime=False, device=True)  # regions and buffers warm
        saturated = run_stream(server, sat_reqs, realtime=False, device=True)
        tiles = [r for r in sat_reqs if r.grid is not None]
        tiles_only = run_stream(server, tiles, realtime=False, device=True)
        host = run_stream(server, sat_reqs, realtime=False, pinned=True)
        pageable = run_stream(server, sat_reqs, realtime=False)
        stats = server.stats()
        # A tile of the stack, served by the same server, against the FP64 oracle (the
        # reference's diamond-square over FP64 posts, craters in double).
        probe_grid = GridSpec(*[int(v) if i < 2 else float(v) for i, v in
                                enumerate(np.load(FP64_FIXTURE)["served_refined_grid"])])
        probe = np.empty(probe_grid.cells, np.float32)
        server.submit_tile(1 << 30, probe_grid, probe)
        server.drain()
        fp64 = {"tile": "257^2 at 0.5 m near the origin (the reference's diamond-square keys "
                        "draws by its raster's posts, which start at the origin)",
                **fp64_error(probe, "served_refined")}
    # The fBm-at-every-cell stack 1e6 m out against the FP64 oracle (the source's far-coordinate
    # precision, which the refined stack's posts share).
    with Server(dev, dem_stack_options(slots=1, refine=False)) as fbm:
        far_grid = GridSpec(*[int(v) if i < 2 else float(v) for i, v in
                              enumerate(np.load(FP64_FIXTURE)["served_grid"])])
        far = np.empty(far_grid.cells, np.float32)
        fbm.submit_tile(1 << 30, far_grid, far)
        fbm.drain()
        fp64_far = {"tile": "257^2 at 0.5 m, 1e6 m out, fBm at every cell",
                    **fp64_error(far, "served")}
    # The plain per-request path on the stream's tile requests (crater records per tile built
    # and resident before timing): the posts of the tile's window, the refinement, the craters.
    sample = tiles[:300]
    prep = []
    ro = refine_options()
    lattice = post_lattice()
    for r in sample:
        g = r.grid
        col0 = int(np.floor(g.x0 / POST_SPACING)) - 8
        row0 = int(np.floor(-g.y0 / POST_SPACING)) - 8
        pw = int(np.ceil((g.x0 + g.width * g.pixel) / POST_SPACING)) + 9 - col0
        ph = int(np.ceil(-(g.y0 - g.height * g.pixel) / POST_SPACING)) + 9 - row0
        window = GridSpec(pw, ph, lattice.x0 + col0 * POST_SPACING,
                          lattice.y0 - row0 * POST_SPACING, POST_SPACING)
        k, rec, dat, foot = crater_batch(opts.craters, g)
        prep.append((g, window, (col0, row0), k, torch.from_numpy(rec.view(np.uint8).copy()).cuda(),
                     torch.from_numpy(np.ascontiguousarray(dat)).cuda(),
                     torch.from_numpy(np.ascontiguousarray(foot)).cuda(), len(rec),
                     torch.empty((ph, pw), dtype=torch.float32, device="cuda"),
                     torch.empty((g.height, g.width), dtype=torch.float32, device="cuda")))

    def plain():
        for g, window, at, k, rec, dat, foot, n, posts, h in prep:
            dev.noise_source(opts._fractals, window, posts, 0.0)
            dev.ds_refine(posts, lattice, g, h, ro.fractal_dimension, ro.scale, seed=ro.seed,
                          window=at)
            if n:
                dev.craters_apply(k, rec, dat, g, h, footprints=foot)

    plain()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plain()
    e1.record()
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    plain_value = sum(r.cells for r in sample) / plain_ms / 1e3
    sat = saturated.summary()
    tonly = tiles_only.summary()
    return {
        "workload": "camera stream at 10 km over a 1737.4 km sphere (planar polar frame, nadir "
                    "1e6 m out): Poisson 2000 req/s, 70% 257^2 / 25% 1025^2 tiles at 0.25-4 m, "
                    "5% x 10,000 points; DEM-refinement stack: 12-octave fBm (20 km, +-2000 m) "
                    "at 5 m posts refined by diamond-square (F 2.2, scale 1.5 m, bilinear) to "
                    "each request's spacing, + craters (2M per 20481^2 at 0.5 m, D 1-100 m)",
        "nominal": nominal.summary(),
        "saturated_device": sat,
        "tiles_only_device": tonly,
        "saturated_host": {"mcells_per_s": host.summary()["mcells_per_s"],
                           "note": "heights copied by the slots' streams straight into "
                                   "page-locked host arrays"},
        "saturated_host_pageable": {"mcells_per_s": pageable.summary()["mcells_per_s"],
                                    "note": "pageable host arrays: through the slots' pinned "
                                            "mirrors and a host copy each"},
        "plain_per_request": {"value": round(plain_value, 3), "unit": UNIT,
                              "requests": len(sample), "ms": round(plain_ms, 3),
                              "path": "tg_noise_source on the tile's post window + "
                                      "tg_ds_refine_window + tg_craters_apply per tile request"},
        "speedup_vs_plain": {"mixed": round(sat["mcells_per_s"] / plain_value, 2),
                             "tiles": round(tonly["mcells_per_s"] / plain_value, 2)},
        "server": {k: stats[k] for k in ("batches", "regions_built", "regions_resident",
                                         "feature_bytes", "peak_bytes", "deferred")},
        "fp64": fp64,
        "fp64_far_source": fp64_far,
        "accuracy": "results identical alone and in the mix; a refined tile is tg_ds_refine_window "
                    "over the same posts bit for bit (tests/test_serve_gpu.py)",
    }


def dem_accuracy(dev):
    """The DEM form's steps against the reference's FP64 computations on their fixtures
    (tests/golden/ds.npz, chain.npz): diamond-square refinement (the reference's nodes are FP64,
    read to float) and the Height seam chain of four patches (the reference's FP64 MG-PCG field)."""
    import torch

    from terraingen_b200.chain import PatchChain, Seams, Window
    from terraingen_b200.device import GridSpec

    def grid_of(row):
        return GridSpec(int(row[0]), int(row[1]), float(row[2]), float(row[3]), float(row[4]))

    def error(got, want):
        err = np.abs(np.asarray(got, np.float64) - want)
        ok = np.isfinite(err)
        return {"max_err_m": float(err[ok].max()), "rms_err_m": float(np.sqrt(np.mean(err[ok] ** 2))),
                "cells": int(ok.sum())}

    out = {}
    ds = np.load(ROOT / "tests" / "golden" / "ds.npz")
    for name in ("dem5m", "tenfold", "tenfold_cr"):
        pg, g = grid_of(ds[f"{name}_post_grid"]), grid_of(ds[f"{name}_grid"])
        fd, scale, seed, interp = ds[f"{name}_options"]
        h = np.zeros((g.height, g.width), np.float32)
        dev.ds_refine(ds[f"{name}_posts"], pg, g, h, fd, scale, int(seed), int(interp))
        out[f"diamond_square_{name}"] = error(h, ds[f"{name}_expected"])
    z = np.load(ROOT / "tests" / "golden" / "chain.npz")
    g = grid_of(z["grid"])
    wins = [Window(*(int(x) for x in w)) for w in z["windows"]]
    _, width, decay = z["height_options"]
    chain = PatchChain(dev, g, wins, Seams("height", width=float(width), decay_length=float(decay)))
    got = chain.compose([torch.from_numpy(z[f"patch{k}"]).cuda() for k in range(4)])
    out["height_seam_chain"] = error(got.cpu().numpy(), z["height_heights"])
    out["against"] = ("the reference CPU path: FP64 diamond-square nodes and FP64 MG-PCG seam "
                      "fields, read to float (fixtures of its own runs)")
    return out


def e2e_leg(dev, w, args, world, device_heights):
    """The e2e leg (see main). Returns the line's `e2e` object plus "_same": whether the last
    step's heights are the device-resident path's bits (`device_heights`)."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from terraingen_b200 import Device
    from terraingen_b200.workloads import DeviceTerrainPrep

    prep_thread = ThreadPoolExecutor(max_workers=1)
    boulder_thread = ThreadPoolExecutor(max_workers=1)

    # Record building on a second handle of the same GPU (its own stream and scratch), so the
    # next step's batch is made while this step evaluates.
    builder = Device(0)
    side, main = torch.cuda.Stream(), torch.cuda.Stream()
    preps = [DeviceTerrainPrep(w.grid, builder, side), DeviceTerrainPrep(w.grid, builder, side)]
    heights = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32, device="cuda")
    h_heights = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32).pin_memory()
    prep_ms, eval_ms = [], []

    def build(q):
        t = time.perf_counter()
        out = preps[q].run(boulder_thread)
        prep_ms.append((time.perf_counter() - t) * 1e3)
        return out

    def run(steps):
        # One long-lived preparing thread (the library keeps its working arrays per thread).
        ahead = prep_thread.submit(build, 0)
        for i in range(steps):
            inputs = ahead.result()
            if i + 1 < steps:
                ahead = prep_thread.submit(build, (i + 1) % 2)
            kernel, rec, data, foot, stones = inputs
            t = time.perf_counter()
            with torch.cuda.stream(main):
                dev.evaluate(w.grid, heights, fractals=w.fractals, elevation=w.elevation,
                             craters=(kernel, rec, data, foot), boulders=stones,
                             boulder_width=w.boulder_width)
                h_heights.copy_(heights, non_blocking=True)
            main.synchronize()
            eval_ms.append((time.perf_counter() - t) * 1e3)
        ahead.result()

    try:
        run(args.warmup)
        prep_ms.clear()
        eval_ms.clear()
        barrier(world)
        t0 = time.perf_counter()
        run(args.steps)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    finally:
        prep_thread.shutdown()
        boulder_thread.shutdown()
        builder.close()
    h2d = preps[0].staged_bytes + w.fractals.nbytes + 188  # + the CraterShapeKernel
    return {"value": round(world * w.cells * args.steps / e2e_s / 1e6, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(w.cells * 4),
            "includes": "every step: crater population, wall terraces and massif peaks on "
                        f"{os.cpu_count()} host threads, then the apply order, the records, their "
                        "data and footprints made on the device (tg_crater_batch_device, its plan "
                        "copied in from page-locked memory), boulder placement (tg_boulder_generate) "
                        "on the host and copied in, tg_evaluate on the device and the heights "
                        "copied out to page-locked memory; the next step's batch is made while "
                        "this step evaluates",
            "host_prep_ms": round(float(np.median(prep_ms)), 3),
            "evaluate_ms": round(float(np.median(eval_ms)), 3),
            "_same": bool(np.array_equal(h_heights.numpy().view(np.uint32),
                                         device_heights.cpu().numpy().view(np.uint32)))}


def e2e_host_records_leg(dev, w, args, world, device_heights):
    """The e2e leg with the crater records made on the host (tg_crater_batch) and every layer
    input passed to tg_evaluate as host buffers; reported beside the e2e line for comparison."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from terraingen_b200.workloads import TerrainPrep

    prep_thread = ThreadPoolExecutor(max_workers=1)

    def pinned(n, dtype):
        return torch.empty(n * np.dtype(dtype).itemsize, dtype=torch.uint8).pin_memory() \
            .numpy().view(dtype)

    preps = [TerrainPrep(w.grid, alloc=pinned), TerrainPrep(w.grid, alloc=pinned)]
    h_heights = torch.empty((w.grid.height, w.grid.width), dtype=torch.float32).pin_memory()
    h_out = h_heights.numpy()
    prep_ms, eval_ms = [], []

    def build(q):
        t = time.perf_counter()
        out = preps[q].run()
        prep_ms.append((time.perf_counter() - t) * 1e3)
        return out

    def run(steps):
        # One long-lived preparing thread (the library keeps its working arrays per thread).
        ahead = prep_thread.submit(build, 0)
        for i in range(steps):
            inputs = ahead.result()
            if i + 1 < steps:
                ahead = prep_thread.submit(build, (i + 1) % 2)
            kernel, rec, data, foot, stones = inputs
            t = time.perf_counter()
            dev.evaluate(w.grid, h_out, fractals=w.fractals, elevation=w.elevation,
                         craters=(kernel, rec, data, foot), boulders=stones,
                         boulder_width=w.boulder_width)
            eval_ms.append((time.perf_counter() - t) * 1e3)
        ahead.result()

    run(args.warmup)
    prep_ms.clear()
    eval_ms.clear()
    barrier(world)
    t0 = time.perf_counter()
    run(args.steps)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    prep_thread.shutdown()
    nr, nd, nb = preps[0].counts
    h2d = nr * (144 + 24) + nd * 4 + nb * 40
    return {"value": round(world * w.cells * args.steps / e2e_s / 1e6, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(w.cells * 4),
            "includes": "every step: crater population, apply order and records "
                        "(tg_crater_batch) and boulder placement (tg_boulder_generate) on "
                        f"{os.cpu_count()} host threads into pinned buffers, then tg_evaluate "
                        "with host buffers (inputs in, heights out); the next step's host work "
                        "overlaps this step's evaluation",
            "host_prep_ms": round(float(np.median(prep_ms)), 3),
            "evaluate_ms": round(float(np.median(eval_ms)), 3),
            "_same": bool(np.array_equal(h_out.view(np.uint32),
                                         device_heights.cpu().numpy().view(np.uint32)))}


def dropin_leg(window):
    """The reference's own Terrain::Evaluate on the reference arm's window, with Backend::Cuda
    served by this library (oracle/_ref/libtgref_cuda.so: the reference's pipeline with crater
    shaping through the drop-in device's tg_craters_apply_lists, and its synthetic source and
    boulder domes through tg_noise_source and tg_boulders_bake; the crater population, records and
    boulder list stay on its CPU path) against Backend::Cpu of the reference's own build."""
    from oracle import harness as H
    from terraingen_b200.workloads import terrain4097_reference_scene

    if not H.available("libtgref_cuda.so"):
        return {"unavailable": "oracle/_ref/libtgref_cuda.so is not built"}
    grid, fr, craters, boulders = terrain4097_reference_scene(window, PIXEL)
    scene = H.make_scene(grid, source_fractals=fr, craters=craters, boulders=boulders)
    lib = H.dropin()
    cpu = H.reference()
    out = {}
    for name, l, backend in (("cuda", lib, 1), ("cpu", cpu, 0)):
        H.evaluate(l, scene, backend, 0)
        times = [H.evaluate(l, scene, backend, 0)[1] for _ in range(3)]
        out[name] = float(np.median(times))
    a, _ = H.evaluate(lib, scene, 1, 0)
    b, _ = H.evaluate(cpu, scene, 0, 0)
    return {"workload": f"{grid.width}x{grid.height} window of terrain4097 through the "
                        "reference's Terrain::Evaluate",
            "cuda_mcells_per_s": round(grid.cells / (out["cuda"] * 1e-3) / 1e6, 3),
            "cpu_mcells_per_s": round(grid.cells / (out["cpu"] * 1e-3) / 1e6, 3),
            "speedup": round(out["cpu"] / out["cuda"], 3),
            "max_abs_diff_m": float(np.abs(a.astype(np.float64) - b).max()),
            "on_gpu": "fBm source (tg_noise_source), crater shaping (RunKernel -> "
                      "tg_craters_apply_lists), boulder domes (tg_boulders_bake)",
            "cores": os.cpu_count()}


def spawn_ranks(n):
    """`--gpus N` (N > 1) started without torchrun: the same command as N ranks on this node under
    torch.distributed.run (rendezvous on 127.0.0.1, a free port); returns their exit status."""
    import socket
    import subprocess

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()),
           *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    rank, world, local = dist_setup(args.gpus)
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but {world} ranks were started")
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
    if args.batched_only:
        form = batched_form(dev, args, rank, world, dev.measure_alu())
        if rank == 0:
            print(json.dumps({"form": "batched", **form}), flush=True)
        return
    if args.served_only:
        form = served_form(dev, args, rank, world)
        if rank == 0:
            print(json.dumps({"form": "served", **form}), flush=True)
        return
    if args.dem_only:
        form = dem_form(dev, args, rank, world)
        if rank == 0:
            print(json.dumps({"form": "dem_refinement", **form}), flush=True)
        return
    # Each rank's own tile, side by side along x (independent tiles, no exchange).
    w = terrain4097(SIDE, PIXEL, cx=ranks.terrain_center(rank, SIDE, PIXEL)[0])
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

    # End to end through the public C ABI from the layers' definitions: every step builds the
    # crater batch (population, apply order, terraces and peaks on the host threads, the records
    # on the device: tg_crater_batch_device) and places the boulders (tg_boulder_generate), then
    # evaluates (tg_evaluate) and copies the heights out. The next step's batch is made on a
    # second thread while this step evaluates, two sets of buffers in turn. The same with the
    # records made on the host and every input passed as host buffers follows for comparison.
    e2e = e2e_leg(dev, w, args, world, heights)
    same = e2e.pop("_same")
    host_records = e2e_host_records_leg(dev, w, args, world, heights)
    same = same and host_records.pop("_same")
    e2e["host_records"] = {k: host_records[k] for k in ("value", "host_prep_ms", "evaluate_ms",
                                                         "h2d_bytes_per_step")}
    e2e_value = e2e["value"]
    # The timed tile's center 257^2 window against the FP64 oracle (rank 0's tile is centered
    # on the origin, as the fixture's window is).
    lo = (SIDE - 257) // 2
    fp64 = {"window": "257^2 at the tile's center",
            **fp64_error(heights.cpu().numpy(), "terrain", slice(lo, lo + 257),
                         slice(lo, lo + 257))}
    forms = {}
    if args.tiles > 0:
        forms["batched"] = batched_form(dev, args, rank, world, alu_peak)
    if args.serve_seconds > 0:
        forms["served"] = served_form(dev, args, rank, world)
    if args.dem_steps > 0:
        forms["dem_refinement"] = dem_form(dev, args, rank, world)
    if args.dem_steps > 0:
        forms["next_rows"] = next_rows_form(dev)

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
    # noise; craters: footprints, pair scan, count, bin scan, lean records, scatter, lean shape,
    # extras pass; boulders: count, bin scan, scatter, bake.
    launches = (1 + (6 + scan_launches(len(w.crater_records)) + scan_launches(nbins)) +
                (3 + scan_launches(nbins)))
    cpu_value, cpu_per, cpu_n, cpu_grid = cpu_sample(1, 1, args.cpu_window)
    dropin = dropin_leg(args.cpu_window)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded): fBm source, the reference's crater batch and boulders "
                "(restated on the host, bit-exact)",
        "config": {"workload": "terrain4097: 4097x4097 at 0.5 m, 8-octave fBm + 200k craters "
                               "(5% central peaks: complex profile from 4.47 m, massif peaks; "
                               "terraces from 200 m on the freshest 10%) + 1M boulders "
                               "(resolved ones drawn)",
                   "cells_per_gpu": w.cells, "craters_on_tile": int(len(w.crater_records)),
                   "boulders_drawn": int(len(w.boulders)), "l2": "flushed between steps",
                   "parallelism": f"replicas x{world} (one tile per GPU)"},
        "phases_ms": {"noise": round(noise_ms, 4), "craters": round(crater_ms, 4),
                      "boulders": round(boulder_ms, 4)},
        "roofline": {"kernel": kernel_name, "bound": "alu",
                     "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "Tops/s",
                     "frac": round(achieved / peak, 3) if peak else None,
                     "peak_source": "tg_measure_alu on this GPU: 4 quadratic IMAD and 4 FFMA "
                                    "dependent chains per thread that no compiler can shorten, "
                                    "thread instructions per second (below the 128 lanes per SM "
                                    "per clock issue ceiling)",
                     "issue": {"thread_inst_per_pair": CRATER_THREAD_INST_PER_PAIR,
                               "achieved": round(counters["crater_pairs"] *
                                                 CRATER_THREAD_INST_PER_PAIR /
                                                 (crater_ms * 1e-3) / 1e12, 3),
                               "frac": round(counters["crater_pairs"] * CRATER_THREAD_INST_PER_PAIR
                                             / (crater_ms * 1e-3) / alu_peak, 3),
                               "note": "crater phase (all its kernels) at the measured per-pair "
                                       "instruction count of the lean kernel"},
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
        "fp64": fp64,
        "e2e": {**e2e, "matches_device_path": same},
        "dropin": dropin,
        "gpu_launches": int(launches * args.steps),
        "clocks": clocks.summary(),
        "forms": forms,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
