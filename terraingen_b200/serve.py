"""The served form (tg_server_* in include/tgb200.h): a request server with continuous batching,
and the request stream of the streaming-renderer use case it is measured on.

`Server` submits tile and point-query requests and polls for finished ones. `camera_stream`
generates the requests a camera orbiting at 10 km over a 1737.4 km sphere asks for (planar
coordinates of the polar frame): Poisson arrivals, 70 % 257^2 tiles, 25 % 1025^2 tiles and 5 %
sets of 10,000 scattered points, tiles at a level of detail that coarsens with distance from the
camera's nadir. `run_stream` replays a stream against a server in real time and reports latency
per class and throughput.
"""

from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .device import Device, GridSpec
from .layouts import fractal

MOON_RADIUS = 1737.4e3
ALTITUDE = 10e3
MOON_GM = 4.9048695e12


def dem_stack_options(seed: int = 3, budget_gb: float = 40.0, slots: int = 3,
                      max_batch_cells: int = 24 << 20, variant: int = -1,
                      base_spacing: float = 0.25, point_spacing: float = 0.5,
                      refine: bool = True, refine_seed: int = 7,
                      crater_density: float = 1.0) -> N.ServerOptions:
    """The DEM-refinement stack's layers as a server serves them. The source is its 12-octave fBm
    relief (wavelength 20 km, amplitude 2000 m) sampled at 5 m posts, refined by diamond-square
    (fractal dimension 2.2, i.e. Hurst 0.8; scale 1.5 m; bilinear) to each request's spacing;
    `refine=False` evaluates the fBm at every cell instead. The crater layer: 2,000,000 craters
    expected over 20481^2 cells of 0.5 m (times `crater_density`), N(>D) ~ D^-2 on [1, 100] m,
    uniform ages over 1 Gyr."""
    fr = np.array([fractal(seed=seed, wavelength=20000.0, amplitude=2000.0, octaves=12)])
    area = (20481 * 0.5) ** 2
    c = crater_density * 2e6 / (area * (1.0 ** -2.0 - 100.0 ** -2.0))
    pop = N.Population(seed=seed, sfd_coefficient=c, sfd_exponent=2.0, min_diameter=1.0,
                       max_diameter=100.0, lifetime_gyr=1.0, depth_ratio=0.2, rim_ratio=0.04,
                       cutoff_depth_ratio=0.04, cell_size_factor=16.0, margin_radii=0.0,
                       min_resolved_diameter=0.0)
    opts = N.ServerOptions(fractals=fr.ctypes.data, n_fractals=1, elevation=0.0, craters=pop,
                           shaping=N.Shaping(profile=0, irregular=1), base_spacing=base_spacing,
                           point_spacing=point_spacing, hbm_budget=int(budget_gb * (1 << 30)),
                           max_batch_cells=max_batch_cells, slots=slots, region_cells=1024,
                           variant=variant, post_spacing=POST_SPACING if refine else 0.0,
                           refine=refine_options(refine_seed))
    opts._fractals = fr  # keep the array alive with the options
    return opts


# The DEM-refinement stack's input DEM: posts every 5 m.
POST_SPACING = 5.0


def refine_options(seed: int = 7) -> N.DsOptions:
    """The DEM refinement's diamond-square options: fractal dimension 2.2 (Hurst 0.8), scale
    1.5 m, bilinear reads."""
    return N.DsOptions(fractal_dimension=2.2, scale=1.5, interp=0, seed=seed, min_pixel_size=0.0)


def post_lattice() -> GridSpec:
    """The served DEM's post lattice as a grid: post (i, j) centered at (i, -j) * 5 m."""
    return GridSpec(1, 1, -0.5 * POST_SPACING, 0.5 * POST_SPACING, POST_SPACING)


class Server:
    """tg_server: submit requests, poll for the finished ones."""

    def __init__(self, device: Device, options: N.ServerOptions):
        self._lib = N.library()
        self._device = device
        self._options = options
        handle = C.c_void_p()
        N.check(self._lib.tg_server_create(device._handle, C.byref(options), C.byref(handle)))
        self._handle = handle
        self._keep = {}
        self._ids = np.zeros(4096, np.uint64)

    def close(self) -> None:
        if self._handle:
            self._lib.tg_server_destroy(self._handle)
            self._handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _out(out, n: int):
        """(pointer, memory) of a float32 output: a numpy array (host) or a torch CUDA tensor."""
        if type(out).__module__.startswith("torch"):
            if not out.is_cuda or not out.is_contiguous() or out.numel() != n or \
                    str(out.dtype) != "torch.float32":
                raise TypeError("out must be a contiguous float32 CUDA tensor of the result")
            return out.data_ptr(), N.TG_MEMORY_DEVICE
        if out.dtype != np.float32 or out.size != n or not out.flags.c_contiguous:
            raise TypeError("out must be a contiguous float32 array of the result")
        return out.ctypes.data, N.TG_MEMORY_HOST

    def submit_tile(self, rid: int, grid: GridSpec, out) -> None:
        ptr, memory = self._out(out, grid.cells)
        req = N.Request(id=rid, kind=0, memory=memory, grid=grid.native(), points=None,
                        n_points=0, heights=ptr)
        N.check(self._lib.tg_server_submit(self._handle, C.byref(req)))
        self._keep[rid] = out

    def submit_points(self, rid: int, xy: np.ndarray, out) -> None:
        xy = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
        ptr, memory = self._out(out, len(xy))
        req = N.Request(id=rid, kind=1, memory=memory, grid=N.Grid(), points=xy.ctypes.data,
                        n_points=len(xy), heights=ptr)
        N.check(self._lib.tg_server_submit(self._handle, C.byref(req)))
        self._keep[rid] = out

    def poll(self, wait: bool = False) -> list[int]:
        n = C.c_size_t()
        N.check(self._lib.tg_server_poll(self._handle, int(wait), self._ids.ctypes.data,
                                         len(self._ids), C.byref(n)))
        done = [int(i) for i in self._ids[:min(n.value, len(self._ids))]]
        for rid in done:
            self._keep.pop(rid, None)
        return done

    def drain(self) -> list[int]:
        done = []
        while self._keep:
            done += self.poll(wait=True)
        return done

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(self._lib.tg_server_stats_get(self._handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in N.ServerStats._fields_}


@dataclass
class Req:
    rid: int
    arrival: float          # seconds from the stream's start
    kind: str               # "tile257", "tile1025", "points"
    grid: GridSpec | None = None
    xy: np.ndarray | None = None

    @property
    def cells(self) -> int:
        return self.grid.cells if self.grid is not None else len(self.xy)


def camera_stream(seconds: float, rate: float = 2000.0, seed: int = 5,
                  start=(1.0e6, 0.0), base_spacing: float = 0.25, levels: int = 6,
                  points: int = 10_000) -> list[Req]:
    """Requests of a camera orbiting at 10 km: its nadir moves at the orbit's ground speed from
    `start`; each request is a tile of 257 or 1025 cells on a side, aligned to its level's tile
    grid, at a distance of up to 10 km (level k = log2(1 + d / 500 m), spacing base * 2^k), or
    `points` points within 5 km of the nadir. Poisson arrivals at `rate` per second."""
    rng = np.random.default_rng(seed)
    speed = math.sqrt(MOON_GM / (MOON_RADIUS + ALTITUDE)) * MOON_RADIUS / (MOON_RADIUS + ALTITUDE)
    reqs, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        nx, ny = start[0], start[1] + speed * t
        u = rng.random()
        theta = rng.uniform(0, 2 * math.pi)
        if u < 0.05:
            r = 5000.0 * np.sqrt(rng.random(points))
            a = rng.uniform(0, 2 * math.pi, points)
            xy = np.stack([nx + r * np.cos(a), ny + r * np.sin(a)], axis=1)
            reqs.append(Req(rid, t, "points", xy=xy))
        else:
            side = 257 if u < 0.75 else 1025
            d = 10000.0 * rng.random() ** 2
            k = min(levels - 1, int(math.log2(1.0 + d / 500.0)))
            pixel = base_spacing * 2 ** k
            span = side * pixel
            cx, cy = nx + d * math.cos(theta), ny + d * math.sin(theta)
            x0 = math.floor(cx / span) * span
            y0 = (math.floor(cy / span) + 1) * span
            reqs.append(Req(rid, t, "tile257" if side == 257 else "tile1025",
                            grid=GridSpec(side, side, x0, y0, pixel)))
        rid += 1
    return reqs


@dataclass
class StreamResult:
    seconds: float
    cells: int
    latency_ms: dict = field(default_factory=dict)   # class -> array of latencies
    outputs: dict = field(default_factory=dict)      # rid -> heights

    def summary(self) -> dict:
        out = {"seconds": round(self.seconds, 4), "cells": self.cells,
               "mcells_per_s": round(self.cells / self.seconds / 1e6, 3)}
        for kind, lat in sorted(self.latency_ms.items()):
            lat = np.asarray(lat)
            out[kind] = {"n": int(len(lat)), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                         "p99_ms": round(float(np.percentile(lat, 99)), 3),
                         "max_ms": round(float(lat.max()), 3)}
        return out


def run_stream(server: Server, reqs: list[Req], realtime: bool = True,
               keep: bool = False, device: bool = False, pinned: bool = False) -> StreamResult:
    """Submits each request at its arrival time (all at once when not `realtime`), polling in
    between; latency is completion minus arrival. Results go to host arrays (page-locked with
    `pinned`, which the server copies into directly), or with `device` to CUDA tensors, all
    allocated before the stream starts."""
    if device:
        import torch

        outs = {r.rid: torch.empty(r.cells, dtype=torch.float32, device="cuda") for r in reqs}
    elif pinned:
        import torch

        outs = {r.rid: torch.empty(r.cells, dtype=torch.float32, pin_memory=True).numpy()
                for r in reqs}
    else:
        outs = {r.rid: np.empty(r.cells, np.float32) for r in reqs}
    arrival = {r.rid: r.arrival for r in reqs}
    kind = {r.rid: r.kind for r in reqs}
    lat: dict = {}
    pending = len(reqs)
    i = 0
    t0 = time.perf_counter()
    while pending:
        now = time.perf_counter() - t0
        while i < len(reqs) and (not realtime or reqs[i].arrival <= now):
            r = reqs[i]
            if r.grid is not None:
                server.submit_tile(r.rid, r.grid, outs[r.rid])
            else:
                server.submit_points(r.rid, r.xy, outs[r.rid])
            if not realtime:
                arrival[r.rid] = now
            i += 1
        done = server.poll(wait=(i == len(reqs)))
        now = time.perf_counter() - t0
        for rid in done:
            lat.setdefault(kind[rid], []).append((now - arrival[rid]) * 1e3)
        pending -= len(done)
    seconds = time.perf_counter() - t0
    res = StreamResult(seconds, sum(r.cells for r in reqs), lat)
    if keep:
        res.outputs = outs
    return res
