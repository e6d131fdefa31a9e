"""Python face of the C ABI: a `Device` whose methods mirror the reference's backend entry points
(RunKernel for noise layers and craters, SyntheticSource::FillSamples, and the CPU-only stages).

Buffers are numpy arrays (host memory: copied in and out inside the call, as RunKernel does) or
torch CUDA tensors (device memory: stream-ordered on torch's current stream, no copies).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .layouts import CRATER_RECORD, CRATER_SHAPE_KERNEL, FRACTAL, NOISE_LAYER_KERNEL


@dataclass(frozen=True)
class GridSpec:
    """A north-up grid: `width` x `height` cells of `pixel` meters, its top-left corner at
    (`x0`, `y0`); row 0 is north (GeoTransform::NorthUp, geo_transform.h:33)."""

    width: int
    height: int
    x0: float
    y0: float
    pixel: float

    def native(self) -> N.Grid:
        return N.Grid(self.width, self.height, self.x0, self.pixel, 0.0, self.y0, 0.0, -self.pixel)

    def transform(self) -> tuple:
        """GDAL-order coefficients."""
        return (self.x0, self.pixel, 0.0, self.y0, 0.0, -self.pixel)

    @property
    def cells(self) -> int:
        return self.width * self.height


def centered(width: int, height: int, pixel: float, cx: float = 0.0, cy: float = 0.0) -> GridSpec:
    """A grid of `width` x `height` cells of `pixel` meters centered on (cx, cy)."""
    return GridSpec(width, height, cx - 0.5 * pixel * width, cy + 0.5 * pixel * height, pixel)


def geographic_sphere_keys(radius: float):
    """GeographicSphereKeys (src/raster/geotiff/geotiff.cpp:103): the GeoKeys of longitude and
    latitude in degrees on a sphere of `radius` meters, as (directory, doubles, ascii)."""
    if not (radius > 0.0 and np.isfinite(radius)):
        raise ValueError("A sphere's radius must be positive and finite")
    user, params = 32767, 34736
    entries = [(1024, 0, 2), (1025, 0, 1), (2048, 0, user), (2050, 0, user), (2054, 0, 9102),
               (2056, 0, user), (2057, params, 0), (2058, params, 1)]
    directory = [1, 1, 0, len(entries)]
    for key, location, value in entries:
        directory += [key, location, 1, value]
    return directory, [float(radius), float(radius)], ""


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


class _Buffers:
    """Resolves each argument to a pointer and records whether the call is host or device."""

    def __init__(self):
        self.memory = None
        self.keep = []

    def ptr(self, x, dtype=None):
        if x is None:
            return None
        if _is_torch(x):
            if not x.is_cuda:
                raise ValueError("torch tensors must be on the GPU")
            if not x.is_contiguous():
                raise ValueError("tensors must be contiguous")
            self._kind(N.TG_MEMORY_DEVICE)
            return C.c_void_p(x.data_ptr())
        arr = np.asarray(x)
        if dtype is not None and arr.dtype != dtype:
            raise TypeError(f"expected {dtype}, got {arr.dtype}")
        if not arr.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous")
        self._kind(N.TG_MEMORY_HOST)
        self.keep.append(arr)
        return C.c_void_p(arr.ctypes.data)

    def _kind(self, memory):
        if self.memory is None:
            self.memory = memory
        elif self.memory != memory:
            raise ValueError("mix of host arrays and device tensors in one call")


# cudaStreamLegacy: torch's default stream has handle 0, which the C ABI reads as "the device's
# own stream", so it is passed as the legacy default stream's handle instead.
_CUDA_STREAM_LEGACY = 0x1


def _stream(memory):
    if memory == N.TG_MEMORY_DEVICE:
        import torch

        handle = torch.cuda.current_stream().cuda_stream
        return C.c_void_p(handle if handle != 0 else _CUDA_STREAM_LEGACY)
    return None


def _bytes(block: np.ndarray, dtype: np.dtype) -> np.ndarray:
    block = np.ascontiguousarray(block)
    if block.dtype != dtype:
        raise TypeError(f"expected a {dtype.itemsize}-byte block")
    return block


class Device:
    """One B200 (tg_open). Methods raise TgError with the library's message on failure."""

    def __init__(self, ordinal: int = 0):
        self._lib = N.library()
        handle = C.c_void_p()
        N.check(self._lib.tg_open(ordinal, C.byref(handle)))
        self._handle = handle

    def close(self) -> None:
        if self._handle:
            self._lib.tg_close(self._handle)
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

    @property
    def name(self) -> str:
        buf = C.create_string_buffer(256)
        N.check(self._lib.tg_device_name(self._handle, buf, 256))
        return buf.value.decode()

    def set_wait_limit(self, polls: int) -> None:
        """tg_set_wait_limit: polls of a staged copy before the binned crater and boulder
        kernels give up with TG_ERROR_TIMEOUT (2^26 by default; 0 gives up at once)."""
        N.check(self._lib.tg_set_wait_limit(self._handle, polls))

    def synchronize(self) -> None:
        N.check(self._lib.tg_synchronize(self._handle))

    # --- noise ----------------------------------------------------------------------------
    def noise_source(self, fractals: np.ndarray, grid: GridSpec, heights, elevation: float = 0.0):
        """SyntheticSource::FillSamples on `grid` (synthetic_source.cpp:87): heights = elevation +
        the fractal stack. `fractals` is an array of FRACTAL (at most 8)."""
        fr = _bytes(np.atleast_1d(fractals), FRACTAL)
        b = _Buffers()
        h = b.ptr(heights, np.float32)
        g = grid.native()
        N.check(self._lib.tg_noise_source(self._handle, fr.ctypes.data, len(fr), elevation,
                                          C.byref(g), h, b.memory, _stream(b.memory)))
        return heights

    def noise_source_body(self, fractals: np.ndarray, grid: GridSpec, radius: float, heights,
                          elevation: float = 0.0):
        """SyntheticSource on a sphere of `radius` m (SyntheticSource::NoiseAt, FractalStackAt on
        a body): `grid` in degrees of longitude and latitude; heights = elevation + the stack in
        3D at each cell center's position."""
        fr = _bytes(np.atleast_1d(fractals), FRACTAL)
        b = _Buffers()
        h = b.ptr(heights, np.float32)
        g = grid.native()
        N.check(self._lib.tg_noise_source_body(self._handle, fr.ctypes.data, len(fr), elevation,
                                               C.byref(g), radius, h, b.memory,
                                               _stream(b.memory)))
        return heights

    def noise_layer(self, kernel: np.ndarray, grid: GridSpec, heights, origin=(0.0, 0.0),
                    nodata=(0, 0.0)):
        """NoiseLayer's RunKernel (noise_layer.cpp:113): heights += the NoiseLayerKernel stack."""
        k = _bytes(kernel, NOISE_LAYER_KERNEL)
        b = _Buffers()
        h = b.ptr(heights, np.float32)
        g = grid.native()
        N.check(self._lib.tg_noise_layer(self._handle, k.ctypes.data, k.nbytes, C.byref(g),
                                         origin[0], origin[1], h, N.NoData(*nodata), b.memory,
                                         _stream(b.memory)))
        return heights

    def noise_layer_rows(self, kernel: np.ndarray, xs, ys, heights, nodata=(0, 0.0)):
        """The strip form RunKernel binds (kernel.cpp:98-111)."""
        k = _bytes(kernel, NOISE_LAYER_KERNEL)
        b = _Buffers()
        px, py, h = b.ptr(xs, np.float32), b.ptr(ys, np.float32), b.ptr(heights, np.float32)
        N.check(self._lib.tg_noise_layer_rows(self._handle, k.ctypes.data, k.nbytes, px, py,
                                              len(xs), len(ys), h, N.NoData(*nodata), b.memory,
                                              _stream(b.memory)))
        return heights

    def noise_probe(self, xy: np.ndarray, seed: int):
        """The conformance probe: (hashes [n, 4] u32, values [n, 12] f32)."""
        xy = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
        n = len(xy)
        hashes = np.zeros((n, 4), np.uint32)
        values = np.zeros((n, 12), np.float32)
        N.check(self._lib.tg_noise_probe(self._handle, xy.ctypes.data, n, seed,
                                         hashes.ctypes.data, values.ctypes.data,
                                         N.TG_MEMORY_HOST))
        return hashes, values

    # --- whole evaluations ----------------------------------------------------------------
    def evaluate(self, grid: GridSpec, heights, fractals=None, elevation: float = 0.0,
                 noise_layer=None, craters=None, boulders=None, boulder_width: float = 0.0):
        """Terrain::Evaluate of a source + noise / crater / boulder stack (tg_evaluate).
        `craters` is (kernel, records, data[, footprints]); host arrays or device tensors alike,
        as the heights are."""
        b = _Buffers()
        h = b.ptr(heights, np.float32)
        t = N.Terrain()
        keep = []
        if fractals is not None:
            fr = _bytes(np.atleast_1d(fractals), FRACTAL)
            keep.append(fr)
            t.fractals, t.n_fractals = fr.ctypes.data, len(fr)
        t.elevation = elevation
        if noise_layer is not None:
            nl = _bytes(noise_layer, NOISE_LAYER_KERNEL)
            keep.append(nl)
            t.noise_layer = nl.ctypes.data
        if craters is not None:
            k = _bytes(craters[0], CRATER_SHAPE_KERNEL)
            keep.append(k)
            t.crater_kernel = k.ctypes.data
            rec, data = craters[1], craters[2]
            t.crater_records = b.ptr(rec)
            t.n_craters = (rec.numel() if _is_torch(rec) else rec.nbytes) // CRATER_RECORD.itemsize
            t.crater_data = b.ptr(data, np.float32)
            t.n_crater_data = data.numel() if _is_torch(data) else len(data)
            if len(craters) > 3 and craters[3] is not None:
                t.crater_footprints = b.ptr(craters[3], np.float64)
        if boulders is not None:
            t.boulders = b.ptr(boulders)
            t.n_boulders = (boulders.numel() if _is_torch(boulders) else boulders.size) // 5
            t.boulder_width = boulder_width
        g = grid.native()
        N.check(self._lib.tg_evaluate(self._handle, C.byref(t), C.byref(g), h, b.memory,
                                      _stream(b.memory)))
        return heights

    # --- diamond-square -------------------------------------------------------------------
    def ds_refine(self, posts, post_grid: GridSpec, grid: GridSpec, heights,
                  fractal_dimension: float, scale: float, seed: int = 1, interp: int = 0,
                  min_pixel_size: float = 0.0, window=(0, 0)):
        """DiamondSquareUpsampler::FillSamples (diamond_square.cpp:488): `posts` [ph, pw] float32
        on `post_grid`, refined and read at every cell of `grid` into `heights`. With `window`
        (col0, row0), `posts` are the lattice's columns col0.. and rows row0.. and `post_grid` the
        whole lattice's (tg_ds_refine_window)."""
        b = _Buffers()
        if _is_torch(posts):
            ph, pw = posts.shape
        else:
            posts = np.ascontiguousarray(posts, np.float32)
            ph, pw = posts.shape
        pp = b.ptr(posts, np.float32)
        h = b.ptr(heights, np.float32)
        o = N.DsOptions(fractal_dimension, scale, interp, seed, min_pixel_size)
        pg, g = post_grid.native(), grid.native()
        N.check(self._lib.tg_ds_refine_window(self._handle, pp, int(window[0]), int(window[1]),
                                              pw, ph, C.byref(pg), C.byref(o), C.byref(g), h,
                                              b.memory, _stream(b.memory)))
        return heights

    # --- seams ---------------------------------------------------------------------------
    SEAM_MODES = {"none": 0, "feather": 1, "height": 2, "slope": 3}

    def seam_solve(self, data, difference, dx: float, dy: float, mode: str, width: float = 50.0,
                   decay_length: float = 50.0, field=None, levels: int = 4, sweeps: int = 2,
                   coarsest_sweeps: int = 20, tolerance: float = 0.0):
        """BuildSeamField (src/sources/seam_field.cpp:663) on the device from the lattice's
        samples: `data` (uint8, 1 where the earlier source has data) and `difference` (float32,
        earlier minus later, NaN elsewhere), both (height, width). Returns the field's posts
        (float32) and the solve's statistics."""
        b = _Buffers()
        if _is_torch(data):
            height, width_ = data.shape
        else:
            data = np.ascontiguousarray(data, np.uint8)
            difference = np.ascontiguousarray(difference, np.float32)
            height, width_ = data.shape
        if field is None:
            if _is_torch(data):
                import torch

                field = torch.empty((height, width_), dtype=torch.float32, device=data.device)
            else:
                field = np.zeros((height, width_), np.float32)
        dp = b.ptr(data)
        fp = b.ptr(difference)
        out = b.ptr(field)
        opts = N.SeamOptions(self.SEAM_MODES[mode], levels, sweeps, coarsest_sweeps, width,
                             decay_length, tolerance)
        N.check(self._lib.tg_seam_solve(self._handle, dp, fp, width_, height, dx, dy,
                                        C.byref(opts), out, b.memory, _stream(b.memory)))
        st = N.SeamStats()
        N.check(self._lib.tg_seam_stats_get(C.byref(st)))
        return field, {"unknowns": st.unknowns, "levels": st.levels,
                       "iterations": st.iterations, "prepare_ms": st.prepare_ms,
                       "solve_ms": st.solve_ms}

    def seam_fill(self, field, lattice: GridSpec, later, grid: GridSpec, heights,
                  nodata=(1, 0.0), window=None):
        """FillGridGaps (src/sources/source_chain.cpp:167): cells of `heights` holding no data
        take `later` plus the field read at their centers. `window` (col0, row0, width, height)
        limits the cells visited to where `later` can have data."""
        b = _Buffers()
        fp = b.ptr(field, np.float32)
        lp = b.ptr(later, np.float32)
        hp = b.ptr(heights, np.float32)
        lg, g = lattice.native(), grid.native()
        win = None if window is None else np.ascontiguousarray(window, np.uint32)
        N.check(self._lib.tg_seam_fill(self._handle, fp, C.byref(lg), lp, C.byref(g), hp,
                                       N.NoData(*nodata),
                                       None if win is None else C.c_void_p(win.ctypes.data),
                                       b.memory, _stream(b.memory)))
        return heights

    GEOTIFF_COMPRESSION = {"none": 0, "lzw": 1, "deflate": 3}

    def geotiff_write(self, path, bands, grid, nodata=None, geokeys=None,
                      compression: str = "lzw", tile_size: int = 256, big_tiff: bool = False):
        """WriteGeoTiff (src/raster/geotiff/geotiff_write.cpp): `bands` (one raster or a list,
        float32 host arrays or CUDA tensors of grid.height x grid.width) as a tiled float32
        GeoTIFF at `path`. `grid` is a GridSpec or (width, height, GDAL-order transform);
        `nodata` None, NaN or a value; `geokeys` None or (directory, doubles, ascii) as
        geographic_sphere_keys gives them; compression "none", "lzw" (the reference's default)
        or "deflate". The tiles are encoded on the device."""
        if not isinstance(bands, (list, tuple)):
            bands = [bands]
        b = _Buffers()
        ptrs = [b.ptr(x, np.float32) for x in bands]
        if isinstance(grid, GridSpec):
            g = grid.native()
        else:
            width, height, t = grid
            g = N.Grid(int(width), int(height), *[float(v) for v in t])
        for x in bands:
            if tuple(x.shape) != (g.height, g.width):
                raise ValueError(f"band shape {tuple(x.shape)} is not the grid's "
                                 f"{(g.height, g.width)}")
        table = (C.c_void_p * len(ptrs))(*ptrs)
        if nodata is None:
            nd = N.NoData(0, 0.0)
        elif np.isnan(nodata):
            nd = N.NoData(1, 0.0)
        else:
            nd = N.NoData(2, float(nodata))
        keys = None
        if geokeys is not None:
            directory, doubles, ascii_ = geokeys
            d = np.ascontiguousarray(directory, np.uint16)
            dp = np.ascontiguousarray(doubles, np.float64)
            b.keep.extend([d, dp])
            keys = N.GeoKeys(C.c_void_p(d.ctypes.data), len(d), len(dp),
                             C.c_void_p(dp.ctypes.data), (ascii_ or "").encode())
        opts = N.GeotiffOptions(self.GEOTIFF_COMPRESSION[compression], tile_size,
                                int(big_tiff), 0)
        N.check(self._lib.tg_geotiff_write(self._handle, str(path).encode(),
                                           C.cast(table, C.c_void_p), len(ptrs), C.byref(g), nd,
                                           None if keys is None else C.byref(keys),
                                           C.byref(opts), b.memory, _stream(b.memory)))

    def seam_samples(self, earlier, later, grid: GridSpec, col0: int, row0: int, lw: int,
                     lh: int, data=None, difference=None, nodata=(1, 0.0)):
        """SampleSources (src/sources/seam_field.cpp:76) for two rasters on `grid`: the lattice
        of `lw` x `lh` posts from cell (`col0`, `row0`). Returns (data uint8, difference f32),
        both (lh, lw), on the host or the device as the inputs are."""
        if _is_torch(earlier):
            import torch

            if data is None:
                data = torch.empty((lh, lw), dtype=torch.uint8, device=earlier.device)
            if difference is None:
                difference = torch.empty((lh, lw), dtype=torch.float32, device=earlier.device)
        else:
            data = np.zeros((lh, lw), np.uint8) if data is None else data
            difference = np.zeros((lh, lw), np.float32) if difference is None else difference
        b = _Buffers()
        ep = b.ptr(earlier, np.float32)
        lp = b.ptr(later, np.float32)
        dp = b.ptr(data)
        fp = b.ptr(difference)
        g = grid.native()
        N.check(self._lib.tg_seam_samples(self._handle, ep, lp, C.byref(g), col0, row0, lw, lh,
                                          N.NoData(*nodata), dp, fp, b.memory,
                                          _stream(b.memory)))
        return data, difference

    def crater_datums(self, kernel, records, data, band_floats, band_cells, cells, entries,
                      targets, heights, width: int, rows: int, first_row: int = 0):
        """FitDatumsWithKernel's relief (KernelDatumRelief, craters.h:1214-1316): `heights`
        (rows x width lattice points, float32) += the relief of the older craters at each point
        of each target crater's fit footprint. `kernel` is the CraterDatumKernel's bytes (host);
        the rest host arrays (raw bytes for `records`) or device tensors."""
        b = _Buffers()
        # The parameter block is read on the host whatever the memory of the rest.
        k = np.ascontiguousarray(np.asarray(kernel), np.uint8)
        kp = C.c_void_p(k.ctypes.data)
        rp = b.ptr(records)
        n_records = (records.numel() if _is_torch(records) else np.asarray(records).nbytes) // 144
        args = []
        for arr, dtype in ((data, np.float32), (band_floats, np.float32),
                           (band_cells, np.uint32), (cells, np.uint32), (entries, np.uint32),
                           (targets, np.uint32)):
            args.append(b.ptr(arr, None if _is_torch(arr) else dtype))
            args.append(arr.numel() if _is_torch(arr) else len(arr))
        hp = b.ptr(heights, None if _is_torch(heights) else np.float32)
        kbytes = k.nbytes
        N.check(self._lib.tg_crater_datums(self._handle, kp, kbytes, rp, n_records, *args, width,
                                           rows, first_row, hp, b.memory, _stream(b.memory)))
        return heights

    def philox_probe(self, sextets: np.ndarray):
        """(words [n, 4] u32, normals [n] f64) of n (counter x4, key x2) sextets."""
        sextets = np.ascontiguousarray(sextets, np.uint32).reshape(-1, 6)
        n = len(sextets)
        out = np.zeros((n, 4), np.uint32)
        normals = np.zeros(n, np.float64)
        N.check(self._lib.tg_philox_probe(self._handle, sextets.ctypes.data, n, out.ctypes.data,
                                          normals.ctypes.data))
        return out, normals

    def counters(self) -> dict:
        """Pairs evaluated by the last crater shaping and boulder bake (tg_device_counters)."""
        out = np.zeros(2, np.uint64)
        N.check(self._lib.tg_device_counters(self._handle, out.ctypes.data, 2))
        return {"crater_pairs": int(out[0]), "boulder_pairs": int(out[1])}

    def measure_alu(self) -> float:
        """Measured IMAD/FFMA lane operations per second (tg_measure_alu)."""
        out = C.c_double()
        N.check(self._lib.tg_measure_alu(self._handle, C.byref(out)))
        return out.value

    # --- boulders -------------------------------------------------------------------------
    def boulders_bake(self, boulders, grid: GridSpec, heights, width: float, nodata=(0, 0.0)):
        """BoulderLayer's dome relief (boulder_relief.cpp:426-439): `boulders` is [n, 5] float64
        (x, y, diameter, exposed height, weight) or a device tensor of the same bytes; `width` the
        band the domes are averaged over (the spacing)."""
        b = _Buffers()
        if _is_torch(boulders):
            n = boulders.numel() // 5
        else:
            boulders = np.ascontiguousarray(boulders, np.float64).reshape(-1, 5)
            n = len(boulders)
        bp = b.ptr(boulders)
        h = b.ptr(heights, np.float32)
        g = grid.native()
        N.check(self._lib.tg_boulders_bake(self._handle, bp, n, width, C.byref(g), h,
                                           N.NoData(*nodata), b.memory, _stream(b.memory)))
        return heights

    # --- craters --------------------------------------------------------------------------
    def craters_apply(self, kernel: np.ndarray, records, data, grid: GridSpec, heights,
                      footprints=None, nodata=(0, 0.0)):
        """ApplyCraters' shaping with device binning (apply.cpp:339-376). `records` is an array
        of CRATER_RECORD (or a uint8 device tensor of its bytes), `data` float32."""
        k = _bytes(kernel, CRATER_SHAPE_KERNEL)
        b = _Buffers()
        if isinstance(records, np.ndarray) and records.dtype == CRATER_RECORD:
            n = len(records)
            rec = b.ptr(records)
        else:
            n = records.numel() // CRATER_RECORD.itemsize if _is_torch(records) else \
                len(records) // CRATER_RECORD.itemsize
            rec = b.ptr(records)
        nd = data.numel() if _is_torch(data) else len(data)
        dp = b.ptr(data, np.float32)
        fp = b.ptr(footprints, np.float64) if footprints is not None else None
        h = b.ptr(heights, np.float32)
        g = grid.native()
        N.check(self._lib.tg_craters_apply(self._handle, k.ctypes.data, k.nbytes, rec, n, dp, nd,
                                           fp, C.byref(g), h, N.NoData(*nodata), b.memory,
                                           _stream(b.memory)))
        return heights

    def crater_batch(self, population, shaping, grid: GridSpec, records=None, data=None,
                     footprints=None):
        """The crater layer's batch for `grid` with its records made on the device
        (tg_crater_batch_device): `records` a uint8 device tensor of 144-byte records, `data`
        float32 and `footprints` float64 device tensors, or all None for the sizes only. Returns
        (kernel, records, floats): the CraterShapeKernel bytes and the batch's sizes; the bytes
        the call copied to the device are then `last_staged_bytes`."""
        import torch

        kernel = np.zeros((), CRATER_SHAPE_KERNEL)
        ptrs, caps = [], []
        for t, unit in ((records, CRATER_RECORD.itemsize), (data, 1), (footprints, 3)):
            if t is not None and not (_is_torch(t) and t.is_cuda and t.is_contiguous()):
                raise ValueError("outputs must be contiguous device tensors")
            ptrs.append(C.c_void_p(t.data_ptr()) if t is not None else None)
            caps.append(t.numel() // unit if t is not None else 0)
        capacity = min([c for c, t in zip((caps[0], caps[2]), (records, footprints))
                        if t is not None], default=0)
        g = grid.native()
        nr, nd, staged = C.c_size_t(), C.c_size_t(), C.c_size_t()
        handle = torch.cuda.current_stream().cuda_stream
        N.check(self._lib.tg_crater_batch_device(
            self._handle, C.byref(population), C.byref(shaping), C.byref(g), kernel.ctypes.data,
            ptrs[0], capacity, ptrs[1], caps[1], ptrs[2], C.byref(nr), C.byref(nd),
            C.byref(staged), C.c_void_p(handle if handle != 0 else _CUDA_STREAM_LEGACY)))
        self.last_staged_bytes = staged.value
        return kernel, nr.value, nd.value

    def craters_apply_lists(self, kernel, records, data, heads, entries, xs, x_lows, ys, y_lows,
                            heights, first_row=0, nodata=(0, 0.0)):
        """The drop-in strip form (craters.slang via ShapeTilesOnGpu, apply.cpp:174-196)."""
        k = _bytes(kernel, CRATER_SHAPE_KERNEL)
        b = _Buffers()
        args = [b.ptr(records), b.ptr(data, np.float32), b.ptr(heads, np.uint32),
                b.ptr(entries, np.uint32), b.ptr(xs, np.float32), b.ptr(x_lows, np.float32),
                b.ptr(ys, np.float32), b.ptr(y_lows, np.float32), b.ptr(heights, np.float32)]
        n = len(records) if records.dtype == CRATER_RECORD else len(records) // 144
        N.check(self._lib.tg_craters_apply_lists(
            self._handle, k.ctypes.data, k.nbytes, args[0], n, args[1], len(data), args[2],
            len(heads), args[3], len(entries), args[4], args[5], args[6], args[7], len(xs),
            len(ys), first_row, args[8], N.NoData(*nodata), b.memory, _stream(b.memory)))
        return heights
