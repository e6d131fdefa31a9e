"""Generates tests/golden/fp64.npz: FP64 heights of sampled windows of the benchmark's forms, the
reference every output's max and RMS error is reported against.

Run here, where the reference sources are, after `make -C oracle REF=<reference> fp64 restate`:

    python tests/golden/fp64_cases.py

Each case holds its grid and its heights in double: the fBm source from the FP64 restatement
(oracle/restate.cpp: the reference's lattice hashes, positions and arithmetic in double), then the
crater layer from the reference's own crater kernel header compiled in double (oracle/fp64.cpp)
on the crater batch tg_crater_batch builds for the grid (the reference's records, bit for bit),
then the boulder layer's dome in double. The GPU tests and the benchmark evaluate the same
windows through the product and compare.

Cases:
  terrain   the synthetic 4097^2 terrain (fBm, 200,000 craters per tile with the peak and terrace
            mapping, boulders), a 257^2 window at its center;
  tile_k    three tiles of the batched form's 4096 uneven tiles (1/10 density), the farthest from
            the origin among those at most 160 cells wide (up to 1.7e6 m out);
  served    a 257^2 tile of the served form's fBm-at-every-cell stack (12-octave fBm, craters)
            1e6 m out;
  served_refined
            a 257^2 tile of the served form's DEM-refinement stack near the origin: the FP64 fBm
            at the 5 m posts (rounded to float, as a DEM's posts), refined by the reference's own
            diamond-square (FP64 nodes; it keys draws by the node's place in its input raster, so
            the raster starts at post (0, 0) as the served lattice does), then the craters in
            double.
"""

from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import harness as H  # noqa: E402
from terraingen_b200 import workloads as W  # noqa: E402
from terraingen_b200.device import GridSpec, centered  # noqa: E402

OUT = Path(__file__).resolve().parent / "fp64.npz"


def fp64_library() -> C.CDLL:
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libtgfp64.so"))
    lib.f64_craters.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                C.c_double, C.c_void_p]
    lib.f64_boulders.argtypes = [C.c_void_p, C.c_size_t, C.c_double, C.c_uint32, C.c_uint32,
                                 C.c_double, C.c_double, C.c_double, C.c_void_p]
    return lib


def fp64_heights(grid: GridSpec, fractal, craters=None, boulders=None) -> np.ndarray:
    """The grid's heights in double: fBm source, then craters (kernel, records, data,
    footprints), then boulders ([n, 5])."""
    out = np.zeros((grid.height, grid.width), np.float64)
    f = np.atleast_1d(fractal)[0]
    H.restate().rs_fbm_grid_f64(grid.width, grid.height, grid.x0, grid.y0, grid.pixel,
                                int(f["seed"]), float(f["wavelength"]), float(f["amplitude"]),
                                int(f["octaves"]), float(f["lacunarity"]), float(f["gain"]), 0.0,
                                out.ctypes.data)
    lib = fp64_library()
    if craters is not None:
        kernel, records, data, foot = craters
        lib.f64_craters(kernel.ctypes.data, records.ctypes.data, len(records), data.ctypes.data,
                        len(data), foot.ctypes.data, grid.width, grid.height, grid.x0, grid.y0,
                        grid.pixel, out.ctypes.data)
    if boulders is not None and len(boulders):
        b = np.ascontiguousarray(boulders, np.float64)
        lib.f64_boulders(b.ctypes.data, len(b), grid.pixel, grid.width, grid.height, grid.x0,
                         grid.y0, grid.pixel, out.ctypes.data)
    return out


def grid_row(g: GridSpec) -> np.ndarray:
    return np.array([g.width, g.height, g.x0, g.y0, g.pixel], np.float64)


def main() -> None:
    arrays = {}
    # The synthetic terrain's center window.
    w = W.terrain4097(257, 0.5)
    arrays["terrain_grid"] = grid_row(w.grid)
    arrays["terrain_fp64"] = fp64_heights(
        w.grid, w.fractals, (w.crater_kernel, w.crater_records, w.crater_data,
                             w.crater_footprints), w.boulders)
    # Batched tiles far out.
    grids = W.uneven_tile_grids()
    population, stones = W.uneven_tile_layers()
    small = [i for i, g in enumerate(grids) if g.width <= 160]
    far = sorted(small, key=lambda i: -np.hypot(grids[i].x0, grids[i].y0))[:3]
    arrays["tiles_index"] = np.array(far, np.int64)
    fr = np.array([W.fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)])
    for k, i in enumerate(far):
        g = grids[i]
        arrays[f"tile{k}_grid"] = grid_row(g)
        arrays[f"tile{k}_fp64"] = fp64_heights(g, fr, W.crater_batch(population, g),
                                               W.generate_boulders(stones, g))
    # A served tile of the DEM stack.
    from terraingen_b200.serve import dem_stack_options

    opts = dem_stack_options(slots=1, refine=False)
    g = GridSpec(257, 257, 1.0e6 + 1000.0, 2000.0 + 257 * 0.5, 0.5)
    arrays["served_grid"] = grid_row(g)
    arrays["served_fp64"] = fp64_heights(g, opts._fractals, W.crater_batch(opts.craters, g))
    # The served DEM-refinement stack.
    from terraingen_b200.serve import POST_SPACING, post_lattice, refine_options

    opts = dem_stack_options(slots=1)
    g = GridSpec(257, 257, 100.0, -100.0, 0.5)
    n = 64  # posts 0..63 along both axes: 0 to 315 m east and south, the tile well inside
    f = opts._fractals[0]
    posts = np.zeros((n, n), np.float64)
    H.restate().rs_fbm_grid_f64(n, n, -0.5 * POST_SPACING, 0.5 * POST_SPACING, POST_SPACING,
                                int(f["seed"]), float(f["wavelength"]), float(f["amplitude"]),
                                int(f["octaves"]), float(f["lacunarity"]), float(f["gain"]), 0.0,
                                posts.ctypes.data)
    lattice = post_lattice()
    r = refine_options()
    refined, _ = H.diamond_square(H.reference(), posts.astype(np.float32),
                                  GridSpec(n, n, lattice.x0, lattice.y0, POST_SPACING), g,
                                  r.fractal_dimension, r.scale, seed=r.seed)
    out = refined.astype(np.float64)
    kernel, records, data, foot = W.crater_batch(opts.craters, g)
    fp64_library().f64_craters(kernel.ctypes.data, records.ctypes.data, len(records),
                               data.ctypes.data, len(data), foot.ctypes.data, g.width, g.height,
                               g.x0, g.y0, g.pixel, out.ctypes.data)
    arrays["served_refined_grid"] = grid_row(g)
    arrays["served_refined_fp64"] = out
    np.savez_compressed(OUT, **arrays)
    for k, v in arrays.items():
        if k.endswith("_fp64"):
            print(k, v.shape, float(v.min()), float(v.max()))


if __name__ == "__main__":
    main()
