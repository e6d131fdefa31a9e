"""Max and RMS height error against the FP64 oracle (tests/golden/fp64.npz, made by
tests/golden/fp64_cases.py) for sampled windows of the benchmark's forms, each evaluated through
the product: the plain path on the synthetic terrain (fBm, craters with central peaks, boulders),
the batched form on three far-out uneven tiles (up to 1.7e6 m from the origin) and the served form
on a tile of the DEM stack 1e6 m out. The bar is 1e-3 m max (the configurations' tolerance)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, grid_of

pytestmark = pytest.mark.gpu

TOLERANCE_M = 1e-3


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN / "fp64.npz"))


def _check(got, want):
    err = np.abs(np.asarray(got, np.float64).reshape(want.shape) - want)
    assert err.max() <= TOLERANCE_M, (float(err.max()), float(np.sqrt(np.mean(err ** 2))))
    return err


def test_terrain_window_within_1mm_of_fp64(device, fx):
    from terraingen_b200.workloads import terrain4097

    w = terrain4097(257, 0.5)
    assert w.grid == grid_of(fx["terrain_grid"])
    got = np.zeros((257, 257), np.float32)
    device.evaluate(w.grid, got, fractals=w.fractals, elevation=w.elevation,
                    craters=(w.crater_kernel, w.crater_records, w.crater_data,
                             w.crater_footprints),
                    boulders=w.boulders, boulder_width=w.boulder_width)
    err = _check(got, fx["terrain_fp64"])
    assert np.count_nonzero(err) > 0


def test_batched_far_tiles_within_1mm_of_fp64(device, fx):
    # The fixture's tiles are picked from the 4096-tile set; a batch of just those.
    from terraingen_b200.batch import TILE, Batch, TileSet, layout
    from terraingen_b200.layouts import fractal
    from terraingen_b200.workloads import (crater_batch, generate_boulders, uneven_tile_grids,
                                           uneven_tile_layers)

    grids = uneven_tile_grids()
    population, stones = uneven_tile_layers()
    picks = [grids[int(i)] for i in fx["tiles_index"]]
    for k, g in enumerate(picks):
        assert g == grid_of(fx[f"tile{k}_grid"])
    offsets, pitch = layout(picks)
    tiles = np.zeros(len(picks), TILE)
    recs, datas, foots, stones_all = [], [], [], []
    nrec = ndata = nstone = 0
    for i, g in enumerate(picks):
        kernel, rec, dat, foot = crater_batch(population, g)
        b = generate_boulders(stones, g)
        t = tiles[i]
        t["width"], t["height"] = g.width, g.height
        t["origin_x"], t["pixel_width"], t["origin_y"], t["pixel_height"] = (
            g.x0, g.pixel, g.y0, -g.pixel)
        t["height_offset"], t["pitch"] = offsets[i], pitch[i]
        t["crater_begin"], t["crater_count"], t["data_begin"] = nrec, len(rec), ndata
        t["boulder_begin"], t["boulder_count"], t["boulder_width"] = nstone, len(b), g.pixel
        recs.append(rec)
        datas.append(dat)
        foots.append(foot)
        stones_all.append(b)
        nrec, ndata, nstone = nrec + len(rec), ndata + len(dat), nstone + len(b)
    fractals = np.array([fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)])
    ts = TileSet(tiles=tiles, fractals=fractals, elevation=0.0, crater_kernel=kernel,
                 crater_records=np.concatenate(recs), crater_data=np.concatenate(datas),
                 crater_footprints=np.concatenate(foots),
                 boulders=np.ascontiguousarray(np.concatenate(stones_all)), grids=picks)
    out = np.zeros(ts.output_floats, np.float32)
    with Batch(device) as b:
        b.run(ts, out)
    for k, g in enumerate(picks):
        o, p = int(offsets[k]), int(pitch[k])
        got = np.stack([out[o + r * p:o + r * p + g.width] for r in range(g.height)])
        _check(got, fx[f"tile{k}_fp64"])


@pytest.mark.parametrize("case,refine", [("served", False), ("served_refined", True)])
def test_served_tile_within_1mm_of_fp64(device, fx, case, refine):
    # The fBm-at-every-cell stack 1e6 m out, and the DEM-refinement stack (diamond-square over
    # the fBm's posts, the reference's own refinement over FP64 posts as the oracle).
    from terraingen_b200.serve import Server, dem_stack_options

    grid = grid_of(fx[f"{case}_grid"])
    out = np.empty(grid.cells, np.float32)
    with Server(device, dem_stack_options(slots=1, refine=refine)) as s:
        s.submit_tile(3, grid, out)
        assert s.drain() == [3]
    _check(out, fx[f"{case}_fp64"])
