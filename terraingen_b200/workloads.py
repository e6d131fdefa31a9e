"""The evaluation workloads of the benchmark configurations, built with the product's own host
code (no reference library): crater batches through tg_crater_batch and boulders through
tg_boulder_generate (the reference's populations, records and boulders, bit for bit).

Synthetic terrain, 4097 x 4097 at 0.5 m ("terrain4097"): an 8-octave Perlin fBm source
(wavelength 512 m, lacunarity 2, gain 0.5, amplitude 5 m, seed 7); 200,000 craters expected over
the tile, N(>D) ~ D^-2 on [1, 500] m, uniform ages over 1 Gyr, fresh depth 0.2 D and rim 0.04 D
worn by freshness, with the default crater apply (irregular outlines, wall terraces, massif
central peaks); 1,000,000 boulders expected, N(>D) ~ D^-2.5 on [0.2, 3] m, heights 0.5 D, of
which those 2 samples or more across (D > 1 m at 0.5 m, about 1.7 %) are drawn.

The configuration's "5 % with central peaks, 10 % with terraced rims for D > 200 m" is mapped
onto the reference's own options, which key both features by diameter and freshness:
  - central peaks: a ComplexCraterProfile over Fassett-Thomson (lunar shape) whose transition
    diameter leaves 5 % of the D^-2 population on [1, 500] m complex (CONFIG2_TRANSITION, about
    4.47 m); every complex crater gets a central peak (massifs, CraterPeaks' defaults);
  - terraced rims: terraces from 200 m (onset) with the minimum freshness set so that 10 % of
    the craters above 200 m are fresh enough to keep them (freshness is uniform on [0.2, 1]
    under these ages and the 0.04 visibility depth, so 0.92).
"""


from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .device import GridSpec, centered
from .layouts import CRATER_RECORD, CRATER_SHAPE_KERNEL, fractal


@dataclass
class Workload:
    name: str
    grid: GridSpec
    fractals: np.ndarray
    elevation: float
    crater_kernel: np.ndarray
    crater_records: np.ndarray
    crater_data: np.ndarray
    crater_footprints: np.ndarray
    boulders: np.ndarray
    boulder_width: float

    @property
    def cells(self) -> int:
        return self.grid.cells

    def input_bytes(self) -> int:
        """Bytes of layer inputs a host-memory evaluation copies to the device."""
        return (self.crater_records.nbytes + self.crater_data.nbytes +
                self.crater_footprints.nbytes + self.boulders.nbytes)


def crater_population(seed: int, coefficient: float, dmin: float, dmax: float,
                      exponent: float = 2.0) -> N.Population:
    return N.Population(seed=seed, sfd_coefficient=coefficient, sfd_exponent=exponent,
                        min_diameter=dmin, max_diameter=dmax, lifetime_gyr=1.0, depth_ratio=0.2,
                        rim_ratio=0.04, cutoff_depth_ratio=0.04, cell_size_factor=16.0,
                        margin_radii=0.0, min_resolved_diameter=0.0)


def generate_craters(population: N.Population, region) -> dict:
    """The craters `population` draws over `region` (x0, y0, x1, y1 in meters) in the
    reference's order (tg_crater_generate): x, y, diameter, age (Gyr) and id arrays."""
    lib = N.library()
    reg = np.ascontiguousarray(region, np.float64)
    count = C.c_size_t()
    N.check(lib.tg_crater_generate(C.byref(population), reg.ctypes.data, None, None, None, None,
                                   None, 0, C.byref(count)))
    n = count.value
    out = {k: np.empty(n, np.float64) for k in ("x", "y", "diameter", "age")}
    out["id"] = np.empty(n, np.uint64)
    N.check(lib.tg_crater_generate(C.byref(population), reg.ctypes.data,
                                   *[out[k].ctypes.data for k in ("x", "y", "diameter", "age",
                                                                  "id")],
                                   n, C.byref(count)))
    return out


def generate_craters_device(device, population: N.Population, region,
                           tolerance: float = 0.0) -> dict:
    """generate_craters drawn on the device (tg_crater_generate_device), into host arrays."""
    lib = N.library()
    reg = np.ascontiguousarray(region, np.float64)
    count = C.c_size_t()
    N.check(lib.tg_crater_generate_device(device._handle, C.byref(population), reg.ctypes.data,
                                          None, None, None, None, None, 0, C.byref(count),
                                          tolerance, N.TG_MEMORY_HOST, None))
    n = count.value
    out = {k: np.empty(n, np.float64) for k in ("x", "y", "diameter", "age")}
    out["id"] = np.empty(n, np.uint64)
    N.check(lib.tg_crater_generate_device(
        device._handle, C.byref(population), reg.ctypes.data,
        *[out[k].ctypes.data for k in ("x", "y", "diameter", "age", "id")], n, C.byref(count),
        tolerance, N.TG_MEMORY_HOST, None))
    return out


# The configuration's peaks and terraces as reference options (module docstring).
CONFIG2_TRANSITION = (0.05 * (1.0 - 500.0 ** -2.0) + 500.0 ** -2.0) ** -0.5
CONFIG2_TERRACES = (200.0, 65000.0, 0.92)  # onset, full diameter, minimum freshness


def config2_shaping() -> N.Shaping:
    """The synthetic terrain's crater shaping: complex craters over Fassett-Thomson from
    CONFIG2_TRANSITION, the default apply (outlines, terraces, peaks), terraces from 200 m."""
    onset, full, freshness = CONFIG2_TERRACES
    return N.Shaping(profile=2, irregular=1, transition_diameter=CONFIG2_TRANSITION,
                     terrace_onset=onset, terrace_full=full, terrace_min_freshness=freshness)


def crater_batch(population: N.Population, grid: GridSpec, profile: int = 0,
                 irregular: int = 1, shaping: N.Shaping | None = None):
    """(kernel, records, data, footprints) a crater layer hands the kernel for `grid`."""
    lib = N.library()
    if shaping is None:
        shaping = N.Shaping(profile=profile, irregular=irregular)
    g = grid.native()
    nr, nd = C.c_size_t(), C.c_size_t()
    N.check(lib.tg_crater_batch(C.byref(population), C.byref(shaping), C.byref(g), None, None, 0,
                                None, 0, None, C.byref(nr), C.byref(nd)))
    kernel = np.zeros((), CRATER_SHAPE_KERNEL)
    records = np.empty(nr.value, CRATER_RECORD)
    data = np.empty(nd.value, np.float32)
    footprints = np.empty(3 * nr.value, np.float64)
    N.check(lib.tg_crater_batch(C.byref(population), C.byref(shaping), C.byref(g),
                                kernel.ctypes.data, records.ctypes.data, nr.value,
                                data.ctypes.data, nd.value, footprints.ctypes.data,
                                C.byref(nr), C.byref(nd)))
    return kernel, records, data, footprints


def boulder_population(seed: int, coefficient: float, exponent: float = 2.5, dmin: float = 0.2,
                       dmax: float = 3.0, height_ratio=(0.5, 0.5),
                       burial=(0.0, 0.0)) -> N.BoulderPopulation:
    return N.BoulderPopulation(seed=seed, sfd_coefficient=coefficient, sfd_exponent=exponent,
                               min_diameter=dmin, max_diameter=dmax,
                               min_height_ratio=height_ratio[0], max_height_ratio=height_ratio[1],
                               min_burial=burial[0], max_burial=burial[1], fade_start_samples=2.0,
                               fade_end_samples=4.0, cell_size_factor=16.0)


def generate_boulders(population: N.BoulderPopulation, grid: GridSpec) -> np.ndarray:
    """[n, 5] boulders (x, y, diameter, exposed height, weight) the boulder layer draws into
    `grid` (tg_boulder_generate over the grid's bounds grown by half a sample)."""
    lib = N.library()
    half = 0.5 * grid.pixel
    region = np.array([grid.x0 - half, grid.y0 - grid.height * grid.pixel - half,
                       grid.x0 + grid.width * grid.pixel + half, grid.y0 + half], np.float64)
    n = C.c_size_t()
    N.check(lib.tg_boulder_generate(C.byref(population), region.ctypes.data, grid.pixel, None, 0,
                                    C.byref(n)))
    out = np.zeros((n.value, 5), np.float64)
    N.check(lib.tg_boulder_generate(C.byref(population), region.ctypes.data, grid.pixel,
                                    out.ctypes.data, n.value, C.byref(n)))
    return out


def resolution_weight(diameter: np.ndarray, spacing: float) -> np.ndarray:
    """1 - Falloff(D / spacing, 2, 4, smoothstep) (src/layers/fade.cpp:50)."""
    x = diameter / spacing
    t = np.clip((x - 2.0) / 2.0, 0.0, 1.0)
    falloff = np.where(x <= 2.0, 1.0, np.where(x >= 4.0, 0.0, 1.0 - t * t * (3.0 - 2.0 * t)))
    return 1.0 - falloff


def terrain4097(side: int = 4097, pixel: float = 0.5, cx: float = 0.0, cy: float = 0.0,
                seed: int = 7) -> Workload:
    """The synthetic 4097^2 terrain (or a `side`^2 window of it centered at (cx, cy))."""
    full_area = (4097 * pixel) ** 2
    grid = centered(side, side, pixel, cx, cy)
    crater_c = 200000.0 / (full_area * (1.0 ** -2.0 - 500.0 ** -2.0))
    kernel, records, data, footprints = crater_batch(
        crater_population(seed, crater_c, 1.0, 500.0), grid, shaping=config2_shaping())
    boulder_c = 1e6 / (full_area * (0.2 ** -2.5 - 3.0 ** -2.5))
    boulders = generate_boulders(boulder_population(seed, boulder_c), grid)
    return Workload("terrain4097", grid,
                    np.array([fractal(seed=seed, wavelength=512.0, amplitude=5.0, octaves=8)]),
                    0.0, kernel, records, data, footprints, boulders, pixel)


class TerrainPrep:
    """The host work the synthetic terrain's layers do before any shaping, for one grid: the
    crater layer's population, apply order and kernel records (tg_crater_batch) and the boulder
    layer's placement (tg_boulder_generate), written into buffers made once (`alloc`, e.g. a
    pinned allocator) and reused by every `run`. The reference's CraterLayer and BoulderLayer
    redo this work on every Terrain::Evaluate."""

    def __init__(self, grid: GridSpec, seed: int = 7, alloc=np.empty, margin: float = 1.25):
        full_area = (4097 * 0.5) ** 2
        self.grid = grid
        self.population = crater_population(
            seed, 200000.0 / (full_area * (1.0 ** -2.0 - 500.0 ** -2.0)), 1.0, 500.0)
        self.shaping = config2_shaping()
        self.stones = boulder_population(seed, 1e6 / (full_area * (0.2 ** -2.5 - 3.0 ** -2.5)))
        half = 0.5 * grid.pixel
        self.region = np.array([grid.x0 - half, grid.y0 - grid.height * grid.pixel - half,
                                grid.x0 + grid.width * grid.pixel + half, grid.y0 + half],
                               np.float64)
        self._grid = grid.native()
        lib = N.library()
        nr, nd, nb = C.c_size_t(), C.c_size_t(), C.c_size_t()
        N.check(lib.tg_crater_batch(C.byref(self.population), C.byref(self.shaping),
                                    C.byref(self._grid), None, None, 0, None, 0, None,
                                    C.byref(nr), C.byref(nd)))
        N.check(lib.tg_boulder_generate(C.byref(self.stones), self.region.ctypes.data,
                                        grid.pixel, None, 0, C.byref(nb)))
        self.record_capacity = int(nr.value * margin) + 64
        self.data_capacity = int(nd.value * margin) + 64
        self.boulder_capacity = int(nb.value * margin) + 64
        self.kernel = np.zeros((), CRATER_SHAPE_KERNEL)
        self.records = alloc(self.record_capacity * CRATER_RECORD.itemsize, np.uint8)
        self.data = alloc(self.data_capacity, np.float32)
        self.footprints = alloc(3 * self.record_capacity, np.float64)
        self.boulders = alloc(5 * self.boulder_capacity, np.float64)
        self.counts = (0, 0, 0)

    def input_bytes(self) -> int:
        nr, nd, nb = self.counts
        return nr * (CRATER_RECORD.itemsize + 24) + nd * 4 + nb * 40

    def run(self):
        """Builds this grid's crater batch and boulders; returns (kernel, records, data,
        footprints, boulders) as views of the buffers."""
        lib = N.library()
        nr, nd, nb = C.c_size_t(), C.c_size_t(), C.c_size_t()
        N.check(lib.tg_crater_batch(C.byref(self.population), C.byref(self.shaping),
                                    C.byref(self._grid), self.kernel.ctypes.data,
                                    self.records.ctypes.data, self.record_capacity,
                                    self.data.ctypes.data, self.data_capacity,
                                    self.footprints.ctypes.data, C.byref(nr), C.byref(nd)))
        N.check(lib.tg_boulder_generate(C.byref(self.stones), self.region.ctypes.data,
                                        self.grid.pixel, self.boulders.ctypes.data,
                                        self.boulder_capacity, C.byref(nb)))
        if nb.value > self.boulder_capacity:
            raise RuntimeError("boulder buffer too small")
        self.counts = (nr.value, nd.value, nb.value)
        records = self.records[:nr.value * CRATER_RECORD.itemsize].view(CRATER_RECORD)
        return (self.kernel, records, self.data[:nd.value], self.footprints[:3 * nr.value],
                self.boulders[:5 * nb.value].reshape(-1, 5))


class DeviceTerrainPrep:
    """TerrainPrep with the crater records made on the device (tg_crater_batch_device on
    `builder`, ordered on `stream`): the crater layer's population, apply order, terraces and
    peaks on the host threads, its records, data and footprints into device tensors made once;
    the boulder layer's placement (tg_boulder_generate) into a pinned buffer, then copied to a
    device tensor on the same stream. Each `run` ends with the stream synchronized, so its
    outputs are ready for any stream."""

    def __init__(self, grid: GridSpec, builder, stream, seed: int = 7, margin: float = 1.25):
        import torch

        full_area = (4097 * 0.5) ** 2
        self.grid = grid
        self.builder = builder
        self.stream = stream
        self.population = crater_population(
            seed, 200000.0 / (full_area * (1.0 ** -2.0 - 500.0 ** -2.0)), 1.0, 500.0)
        self.shaping = config2_shaping()
        self.stones = boulder_population(seed, 1e6 / (full_area * (0.2 ** -2.5 - 3.0 ** -2.5)))
        half = 0.5 * grid.pixel
        self.region = np.array([grid.x0 - half, grid.y0 - grid.height * grid.pixel - half,
                                grid.x0 + grid.width * grid.pixel + half, grid.y0 + half],
                               np.float64)
        with torch.cuda.stream(stream):
            _, nr, nd = builder.crater_batch(self.population, self.shaping, grid)
        nb = C.c_size_t()
        N.check(N.library().tg_boulder_generate(C.byref(self.stones), self.region.ctypes.data,
                                                grid.pixel, None, 0, C.byref(nb)))
        self.record_capacity = int(nr * margin) + 64
        self.data_capacity = int(nd * margin) + 64
        self.boulder_capacity = int(nb.value * margin) + 64
        cuda = dict(device="cuda")
        self.records = torch.empty(self.record_capacity * CRATER_RECORD.itemsize,
                                   dtype=torch.uint8, **cuda)
        self.data = torch.empty(self.data_capacity, dtype=torch.float32, **cuda)
        self.footprints = torch.empty(3 * self.record_capacity, dtype=torch.float64, **cuda)
        self.boulders = torch.empty(5 * self.boulder_capacity, dtype=torch.float64, **cuda)
        self.host_boulders = torch.empty(5 * self.boulder_capacity,
                                         dtype=torch.float64).pin_memory()
        self.counts = (0, 0, 0)
        self.staged_bytes = 0

    def _place_boulders(self) -> int:
        nb = C.c_size_t()
        N.check(N.library().tg_boulder_generate(
            C.byref(self.stones), self.region.ctypes.data, self.grid.pixel,
            self.host_boulders.data_ptr(), self.boulder_capacity, C.byref(nb)))
        return nb.value

    def run(self, boulder_thread=None):
        """Builds this grid's crater batch and boulders; returns (kernel, records, data,
        footprints, boulders), the last four device tensors (views of the buffers). With
        `boulder_thread` (an executor) the boulders are placed there while the crater batch is
        made."""
        import torch

        placing = boulder_thread.submit(self._place_boulders) if boulder_thread else None
        with torch.cuda.stream(self.stream):
            kernel, nr, nd = self.builder.crater_batch(self.population, self.shaping, self.grid,
                                                       self.records, self.data, self.footprints)
            nb = placing.result() if placing else self._place_boulders()
            if nb > self.boulder_capacity:
                raise RuntimeError("boulder buffer too small")
            stones = self.boulders[:5 * nb]
            stones.copy_(self.host_boulders[:5 * nb], non_blocking=True)
        self.stream.synchronize()
        self.counts = (nr, nd, nb)
        self.staged_bytes = self.builder.last_staged_bytes + 40 * nb
        return (kernel, self.records[:nr * CRATER_RECORD.itemsize], self.data[:nd],
                self.footprints[:3 * nr], stones)


def terrain4097_reference_scene(side: int, pixel: float = 0.5, seed: int = 7):
    """The same terrain as the reference CPU path builds it (oracle harness scene fields)."""
    full_area = (4097 * pixel) ** 2
    crater_c = 200000.0 / (full_area * (1.0 ** -2.0 - 500.0 ** -2.0))
    boulder_c = 1e6 / (full_area * (0.2 ** -2.5 - 3.0 ** -2.5))
    onset, full, freshness = CONFIG2_TERRACES
    craters = dict(seed=seed, sfdCoefficient=crater_c, sfdExponent=2.0, minDiameter=1.0,
                   maxDiameter=500.0, lifetimeGyr=1.0, depthRatio=0.2, rimRatio=0.04, profile=2,
                   transitionDiameter=CONFIG2_TRANSITION, applyPreset=0, terraceOnset=onset,
                   terraceFull=full, terraceMinFreshness=freshness)
    boulders = dict(boulderSeed=seed, boulderCoefficient=boulder_c, boulderExponent=2.5,
                    boulderMin=0.2, boulderMax=3.0, heightRatio=0.5)
    grid = centered(side, side, pixel)
    fr = np.array([fractal(seed=seed, wavelength=512.0, amplitude=5.0, octaves=8)])
    return grid, fr, craters, boulders


def uneven_tile_grids(n: int = 4096, side=(65, 1025), spacing=(0.25, 2.0),
                      radius: float = 1.7e6, seed: int = 11) -> list:
    """The grids of `uneven_tiles` (sides, spacings and centers drawn from `seed`)."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(np.log(side[0]), np.log(side[1] + 1), n)).astype(np.int64)
    sides = np.clip(sides, side[0], side[1])
    pixels = np.exp(rng.uniform(np.log(spacing[0]), np.log(spacing[1]), n))
    r = radius * np.sqrt(rng.random(n))
    theta = rng.uniform(0.0, 2.0 * np.pi, n)
    cxs, cys = r * np.cos(theta), r * np.sin(theta)
    return [centered(int(s), int(s), float(p), float(x), float(y))
            for s, p, x, y in zip(sides, pixels, cxs, cys)]


def uneven_tile_layers(density: float = 0.1):
    """The crater population and boulder sizes of `uneven_tiles` at `density` times the
    synthetic terrain's."""
    full_area = (4097 * 0.5) ** 2
    crater_c = density * 200000.0 / (full_area * (1.0 ** -2.0 - 500.0 ** -2.0))
    population = crater_population(7, crater_c, 1.0, 500.0)
    stones_of = boulder_population(7, density * 1e6 / (full_area * (0.2 ** -2.5 - 3.0 ** -2.5)))
    return population, stones_of


def uneven_tiles(n: int = 4096, side=(65, 1025), spacing=(0.25, 2.0), radius: float = 1.7e6,
                 density: float = 0.1, seed: int = 11, boulders: bool = True):
    """Uneven tiles of the synthetic terrain's stack ("tiles4096"): `n` square tiles with sides
    log-uniform on `side` cells, spacings log-uniform on `spacing` m, centers uniform over a disk
    of `radius` m around the origin (the polar frame of a 1737.4 km sphere), the 4097^2 terrain's
    source, and its craters and boulders at `density` times their density. Each tile carries the
    craters tg_crater_batch builds for its grid and the boulders tg_boulder_generate draws into
    it."""
    from .batch import TILE, TileSet, layout

    grids = uneven_tile_grids(n, side, spacing, radius, seed)
    population, stones_of = uneven_tile_layers(density)
    offsets, pitch = layout(grids)
    tiles = np.zeros(n, TILE)
    kernel = None
    records, data, footprints, stones = [], [], [], []
    nrec = ndata = nstone = 0
    for i, g in enumerate(grids):
        k, rec, dat, foot = crater_batch(population, g)
        kernel = k if kernel is None else kernel
        if boulders:
            b = generate_boulders(stones_of, g)
        else:
            b = np.zeros((0, 5), np.float64)
        t = tiles[i]
        t["width"], t["height"] = g.width, g.height
        t["origin_x"], t["pixel_width"], t["origin_y"], t["pixel_height"] = (
            g.x0, g.pixel, g.y0, -g.pixel)
        t["height_offset"], t["pitch"] = offsets[i], pitch[i]
        t["crater_begin"], t["crater_count"], t["data_begin"] = nrec, len(rec), ndata
        t["boulder_begin"], t["boulder_count"] = nstone, len(b)
        t["boulder_width"] = g.pixel
        records.append(rec)
        data.append(dat)
        footprints.append(foot)
        stones.append(b)
        nrec += len(rec)
        ndata += len(dat)
        nstone += len(b)
    return TileSet(
        tiles=tiles,
        fractals=np.array([fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)]),
        elevation=0.0,
        crater_kernel=kernel if kernel is not None else np.zeros((), CRATER_SHAPE_KERNEL),
        crater_records=np.concatenate(records) if records else np.zeros(0, CRATER_RECORD),
        crater_data=np.concatenate(data).astype(np.float32) if data else np.zeros(0, np.float32),
        crater_footprints=np.concatenate(footprints) if footprints else np.zeros(0),
        boulders=np.ascontiguousarray(np.concatenate(stones)) if stones else np.zeros((0, 5)),
        grids=grids)


@dataclass
class DemRefinement:
    """The DEM refinement ("dem20481"): a 2049^2 float32 DEM at 5 m (12-octave fBm, wavelength
    20 km, amplitude 2000 m) refined 10-fold by diamond-square (F = 2.2, i.e. Hurst 0.8, 4 levels,
    bilinear read) to 20481^2 at 0.5 m as 2 x 2 patches, each its own refinement (its own seed)
    of a quadrant with a 64-cell overlap, chained with Height seams reaching 64 cells (3 L = 32 m);
    then 2,000,000 craters expected over the grid, N(>D) ~ D^-2 on [1, 100] m."""

    post_grid: GridSpec
    fractals: np.ndarray
    grid: GridSpec
    windows: list
    seeds: list
    fractal_dimension: float
    scale: float
    decay_length: float
    crater_kernel: np.ndarray
    crater_records: np.ndarray
    crater_data: np.ndarray
    crater_footprints: np.ndarray

    @property
    def cells(self) -> int:
        return self.grid.cells


def dem20481(side: int = 20481, posts: int = 2049, overlap: int = 64, seed: int = 7,
             craters: float = 2e6, crater_seed: int = 11) -> DemRefinement:
    """The DEM refinement workload (or a smaller one of the same make: `side` output cells a
    side at 0.5 m over `posts` posts at 5 m; craters scale with the area)."""
    from .chain import Window

    post_grid = centered(posts, posts, 5.0)
    grid = centered(side, side, 0.5)
    half = side // 2
    lo, hi = half + overlap // 2, half - overlap // 2
    windows = [Window(0, 0, lo, lo), Window(hi, 0, side - hi, lo),
               Window(0, hi, lo, side - hi), Window(hi, hi, side - hi, side - hi)]
    area = grid.width * grid.height * grid.pixel ** 2
    expected = craters * area / (20481 * 0.5) ** 2
    c = expected / (area * (1.0 ** -2.0 - 100.0 ** -2.0))
    kernel, records, data, footprints = crater_batch(
        crater_population(crater_seed, c, 1.0, 100.0), grid)
    return DemRefinement(post_grid,
                         np.array([fractal(seed=3, wavelength=20000.0, amplitude=2000.0,
                                           octaves=12)]),
                         grid, windows, [seed + k for k in range(4)], 2.2, 1.5,
                         overlap * grid.pixel / 3.0, kernel, records, data, footprints)
