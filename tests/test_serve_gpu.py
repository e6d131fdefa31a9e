"""GPU tests of the served form (tg_server_*): continuous batching of tile and point requests.

The served stack is the DEM refinement's: the 12-octave fBm sampled at 5 m posts, refined by
diamond-square to each request's spacing, craters on top; the fBm-at-every-cell stack
(refine=False) is tested too.

- A request's heights are the same alone (on a fresh server) and in a mix of requests.
- A served refined tile equals tg_ds_refine_window over the same posts bit for bit, and with its
  craters the plain path (refinement, then tg_craters_apply) within 1e-3 m; served points equal
  the refined tile's cells; the refined source is within 1e-3 m of the reference's diamond-square
  over FP64 posts.
- A served tile equals the batch engine's evaluation of the same tile from tg_crater_batch's
  records for its grid (the region split owns every crater that reaches the tile).
- The 2000 m source stays within 1e-3 m of the FP64 oracle 1e6 m from the origin (compensated
  octave sums).
- A small memory budget defers admissions without losing requests.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import harness as H

pytestmark = pytest.mark.gpu


def _stream(seconds=0.03, seed=8, points=2000):
    from terraingen_b200.serve import camera_stream

    return camera_stream(seconds, rate=2000.0, seed=seed, points=points)


def test_served_alone_equals_in_the_mix(device):
    from terraingen_b200.serve import Server, dem_stack_options, run_stream

    reqs = _stream()
    kinds = {r.kind for r in reqs}
    assert {"tile257", "tile1025", "points"} <= kinds, kinds
    with Server(device, dem_stack_options(slots=3, max_batch_cells=4 << 20)) as s:
        mix = run_stream(s, reqs, realtime=False, keep=True)
        st = s.stats()
    assert st["completed"] == len(reqs) and st["batches"] >= 2
    picks = [r for r in reqs if r.kind == "points"][:1] + [r for r in reqs if r.kind != "points"][:6]
    for r in picks:
        with Server(device, dem_stack_options(slots=1)) as alone:
            one = run_stream(alone, [r], realtime=False, keep=True)
        a, b = mix.outputs[r.rid], one.outputs[r.rid]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (
            r.kind, float(np.abs(a.astype(np.float64) - b).max()))


def test_served_tile_equals_batched_tile(device):
    from terraingen_b200.batch import TILE, Batch, TileSet, layout
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options
    from terraingen_b200.workloads import crater_batch

    opts = dem_stack_options(slots=1, refine=False)
    grid = GridSpec(300, 260, 1.0e6 + 1000.0, 250.0 + 260 * 0.5, 0.5)
    out = np.empty(grid.cells, np.float32)
    with Server(device, opts) as s:
        s.submit_tile(1, grid, out)
        assert s.drain() == [1]
    kernel, records, data, foot = crater_batch(opts.craters, grid)
    assert len(records) > 50
    offsets, pitch = layout([grid])
    t = np.zeros(1, TILE)
    t["width"], t["height"] = grid.width, grid.height
    t["origin_x"], t["pixel_width"], t["origin_y"], t["pixel_height"] = (
        grid.x0, grid.pixel, grid.y0, -grid.pixel)
    t["height_offset"], t["pitch"], t["crater_count"] = offsets[0], pitch[0], len(records)
    ts = TileSet(tiles=t, fractals=opts._fractals, elevation=0.0, crater_kernel=kernel,
                 crater_records=records, crater_data=data, crater_footprints=foot,
                 boulders=np.zeros((0, 5)), grids=[grid])
    want = np.zeros(ts.output_floats, np.float32)
    with Batch(device) as b:
        b.run(ts, want)
    got = out.reshape(grid.height, grid.width)
    err = np.abs(got.astype(np.float64) - ts.tile_view(want, 0)).max()
    assert err <= 1e-5, err


def test_served_source_within_1mm_of_fp64(device):
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options

    opts = dem_stack_options(slots=1, refine=False)
    opts.craters.sfd_coefficient = 1e-15  # no craters: the source alone
    grid = GridSpec(257, 257, 1.2e6 + 333.0, -4.0e5 + 64.25, 2.0)
    out = np.empty(grid.cells, np.float32)
    with Server(device, opts) as s:
        s.submit_tile(7, grid, out)
        s.drain()
    f = opts._fractals[0]
    want = np.zeros((grid.height, grid.width), np.float64)
    H.restate().rs_fbm_grid_f64(grid.width, grid.height, grid.x0, grid.y0, grid.pixel,
                                int(f["seed"]), float(f["wavelength"]), float(f["amplitude"]),
                                int(f["octaves"]), float(f["lacunarity"]), float(f["gain"]), 0.0,
                                want.ctypes.data)
    err = np.abs(out.reshape(want.shape).astype(np.float64) - want)
    assert np.abs(want).max() > 100.0
    assert err.max() <= 1e-3, (err.max(), float(np.sqrt(np.mean(err ** 2))))


def test_served_budget_defers_admission(device):
    # 40 tiles of 1025^2 (42M cells) under a 0.6 GB budget: batches are cut by the budget, not by
    # max_batch_cells, and every request still completes. The stream runs twice: on the second
    # pass every region is resident when the requests arrive, so the first batch sees all 40
    # waiting whatever the timing of the region builds.
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Req, Server, dem_stack_options, run_stream

    reqs = [Req(i, 0.0, "tile1025", grid=GridSpec(1025, 1025, 1.0e6 + 512.5 * (i % 8),
                                                  2000.0 + 512.5 * (i // 8), 0.5))
            for i in range(40)]
    opts = dem_stack_options(slots=2, budget_gb=0.6, max_batch_cells=1 << 40)
    with Server(device, opts) as s:
        run_stream(s, [Req(r.rid + len(reqs), 0.0, r.kind, grid=r.grid) for r in reqs],
                   realtime=False)
        res = run_stream(s, reqs, realtime=False)
        st = s.stats()
    assert st["completed"] == 2 * len(reqs)
    assert st["deferred"] > 0 and st["batches"] >= 2
    assert sum(len(v) for v in res.latency_ms.values()) == len(reqs)


def test_served_device_outputs_equal_host_outputs(device):
    import torch

    from terraingen_b200.serve import Server, dem_stack_options, run_stream

    reqs = _stream(0.01, seed=12)
    with Server(device, dem_stack_options(slots=2, max_batch_cells=2 << 20)) as s:
        host = run_stream(s, reqs, realtime=False, keep=True)
        pinned = run_stream(s, reqs, realtime=False, keep=True, pinned=True)
        dev = run_stream(s, reqs, realtime=False, keep=True, device=True)
    for r in reqs:
        a = host.outputs[r.rid]
        b = dev.outputs[r.rid].cpu().numpy()
        c = pinned.outputs[r.rid]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), r.kind
        assert np.array_equal(c.view(np.uint32), b.view(np.uint32)), r.kind


def test_served_points_equal_batched_points(device):
    # Points read their regions' resident cell lists; the batch engine bins the same points
    # against tg_crater_batch's records over their bounding box: the same heights.
    from terraingen_b200.batch import POINT_SET, Batch, TileSet
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options
    from terraingen_b200.workloads import crater_batch

    opts = dem_stack_options(slots=1, refine=False)
    rng = np.random.default_rng(4)
    xy = np.stack([1.0e6 + 300.0 + 1500.0 * rng.random(3000),
                   -2.0e3 + 1200.0 * rng.random(3000)], axis=1)
    out = np.empty(len(xy), np.float32)
    with Server(device, opts) as s:
        s.submit_points(3, xy, out)
        assert s.drain() == [3]
    pixel = opts.point_spacing
    x0, y1 = np.floor(xy[:, 0].min()) - 1, np.ceil(xy[:, 1].max()) + 1
    w = int(np.ceil((xy[:, 0].max() + 1 - x0) / pixel))
    h = int(np.ceil((y1 - xy[:, 1].min() + 1) / pixel))
    kernel, records, data, foot = crater_batch(opts.craters, GridSpec(w, h, x0, y1, pixel))
    sets = np.zeros(1, POINT_SET)
    sets["point_count"], sets["crater_count"] = len(xy), len(records)
    ts = TileSet(tiles=np.zeros(0, __import__("terraingen_b200.batch", fromlist=["TILE"]).TILE),
                 fractals=opts._fractals, elevation=0.0, crater_kernel=kernel,
                 crater_records=records, crater_data=data, crater_footprints=foot,
                 boulders=np.zeros((0, 5)), point_sets=sets, points=xy)
    want = np.zeros(ts.output_floats, np.float32)
    with Batch(device) as b:
        b.run(ts, want)
        assert b.stats()["crater_pairs"] > 0
    err = np.abs(out.astype(np.float64) - want).max()
    assert err <= 1e-5, err


def _posts(device, opts, col0, row0, pw, ph):
    """The served DEM's posts (the lattice's columns col0.. and rows row0..): the batch engine's
    source at each post center (i, -j) * 5 m, as a point set with no craters."""
    from terraingen_b200.batch import POINT_SET, TILE, Batch, TileSet
    from terraingen_b200.serve import POST_SPACING
    from terraingen_b200.layouts import CRATER_RECORD, CRATER_SHAPE_KERNEL

    cols = np.arange(col0, col0 + pw, dtype=np.float64)
    rows = np.arange(row0, row0 + ph, dtype=np.float64)
    xy = np.stack(np.broadcast_arrays(cols[None, :] * POST_SPACING,
                                      -rows[:, None] * POST_SPACING), axis=-1).reshape(-1, 2)
    sets = np.zeros(1, POINT_SET)
    sets["point_count"] = len(xy)
    ts = TileSet(tiles=np.zeros(0, TILE), fractals=opts._fractals, elevation=0.0,
                 crater_kernel=np.zeros((), CRATER_SHAPE_KERNEL),
                 crater_records=np.zeros(0, CRATER_RECORD), crater_data=np.zeros(1, np.float32),
                 crater_footprints=np.zeros(0), boulders=np.zeros((0, 5)), point_sets=sets,
                 points=xy)
    out = np.zeros(ts.output_floats, np.float32)
    with Batch(device) as b:
        b.run(ts, out)
    return out.reshape(ph, pw)


def _window(grid, margin=8):
    """(col0, row0, pw, ph): the post window a tile's refinement reads, with a margin of posts."""
    from terraingen_b200.serve import POST_SPACING

    x1, y0 = grid.x0 + grid.width * grid.pixel, grid.y0 - grid.height * grid.pixel
    col0 = int(np.floor(grid.x0 / POST_SPACING)) - margin
    row0 = int(np.floor(-grid.y0 / POST_SPACING)) - margin
    pw = int(np.ceil(x1 / POST_SPACING)) + margin - col0 + 1
    ph = int(np.ceil(-y0 / POST_SPACING)) + margin - row0 + 1
    return col0, row0, pw, ph


@pytest.mark.parametrize("pixel,x0", [(0.25, 4.0e5 + 3.3), (0.5, -1.0e6 + 127.0),
                                      (2.0, 1.2e6 + 9.0), (8.0, 6.0e5 + 40.0)])
def test_served_refined_tile_is_the_refinement(device, pixel, x0):
    # No craters: the served tile is the diamond-square refinement of the fBm's posts, the same
    # bits as tg_ds_refine_window over the same posts (levels from 5 to 0 as the spacing grows).
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options, post_lattice, refine_options

    opts = dem_stack_options(slots=1)
    opts.craters.sfd_coefficient = 1e-15
    grid = GridSpec(300, 257, x0, -2.5e5 + 51.0, pixel)
    out = np.empty(grid.cells, np.float32)
    with Server(device, opts) as s:
        s.submit_tile(1, grid, out)
        assert s.drain() == [1]
    col0, row0, pw, ph = _window(grid)
    posts = _posts(device, opts, col0, row0, pw, ph)
    r = refine_options()
    want = np.zeros((grid.height, grid.width), np.float32)
    device.ds_refine(posts, post_lattice(), grid, want, r.fractal_dimension, r.scale, seed=r.seed,
                     window=(col0, row0))
    got = out.reshape(want.shape)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), float(
        np.abs(got.astype(np.float64) - want).max())
    assert float(got.std()) > 0.01


def test_served_refined_tile_matches_plain_path(device):
    # With craters: the plain per-request path (tg_ds_refine_window, then tg_craters_apply with
    # tg_crater_batch's records for the tile) within 1e-3 m.
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options, post_lattice, refine_options
    from terraingen_b200.workloads import crater_batch

    opts = dem_stack_options(slots=1)
    grid = GridSpec(320, 256, 2.0e5 + 61.0, 7.0e5 + 3.0, 0.5)
    out = np.empty(grid.cells, np.float32)
    with Server(device, opts) as s:
        s.submit_tile(1, grid, out)
        assert s.drain() == [1]
    col0, row0, pw, ph = _window(grid)
    posts = _posts(device, opts, col0, row0, pw, ph)
    r = refine_options()
    want = np.zeros((grid.height, grid.width), np.float32)
    device.ds_refine(posts, post_lattice(), grid, want, r.fractal_dimension, r.scale, seed=r.seed,
                     window=(col0, row0))
    base = want.copy()
    kernel, records, data, foot = crater_batch(opts.craters, grid)
    assert len(records) > 200
    device.craters_apply(kernel, records, data, grid, want)
    assert np.abs(want.astype(np.float64) - base).max() > 0.1
    err = np.abs(out.reshape(want.shape).astype(np.float64) - want).max()
    assert err <= 1e-3, err


def test_served_refined_points_are_the_tile_cells(device):
    # Points at the point spacing read the same nodes as a tile at that spacing: at its cell
    # centers they give its heights (no craters: the refinement alone, bit for bit).
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options

    opts = dem_stack_options(slots=1)
    opts.craters.sfd_coefficient = 1e-15
    grid = GridSpec(64, 48, -3.0e5 + 17.0, 9.0e5 + 2.0, opts.point_spacing)
    tile = np.empty(grid.cells, np.float32)
    rng = np.random.default_rng(2)
    cells = rng.choice(grid.cells, 500, replace=False)
    cx, cy = cells % grid.width, cells // grid.width
    xy = np.stack([grid.x0 + (cx + 0.5) * grid.pixel, grid.y0 - (cy + 0.5) * grid.pixel], axis=1)
    pts = np.empty(len(xy), np.float32)
    with Server(device, opts) as s:
        s.submit_tile(1, grid, tile)
        s.submit_points(2, xy, pts)
        assert sorted(s.drain()) == [1, 2]
    assert np.array_equal(pts.view(np.uint32), tile[cells].view(np.uint32))


def test_served_refined_source_within_1mm_of_fp64(device):
    # The refined source against the reference's own diamond-square (FP64 nodes) over posts from
    # the FP64 fBm, rounded to float. The reference keys its draws by the node's place in its
    # input raster, so the raster starts at post (0, 0), as the served lattice does, and the tile
    # lies well inside it: max error within 1e-3 m.
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import POST_SPACING, Server, dem_stack_options, post_lattice

    opts = dem_stack_options(slots=1)
    opts.craters.sfd_coefficient = 1e-15
    grid = GridSpec(257, 257, 100.0, -100.0, 0.5)
    out = np.empty(grid.cells, np.float32)
    with Server(device, opts) as s:
        s.submit_tile(1, grid, out)
        s.drain()
    n = 64  # posts 0..63 along both axes: 0 to 315 m east and south
    f = opts._fractals[0]
    posts64 = np.zeros((n, n), np.float64)
    H.restate().rs_fbm_grid_f64(n, n, -0.5 * POST_SPACING, 0.5 * POST_SPACING, POST_SPACING,
                                int(f["seed"]), float(f["wavelength"]), float(f["amplitude"]),
                                int(f["octaves"]), float(f["lacunarity"]), float(f["gain"]), 0.0,
                                posts64.ctypes.data)
    lattice = post_lattice()
    raster = GridSpec(n, n, lattice.x0, lattice.y0, POST_SPACING)
    want, _ = H.diamond_square(H.reference(), posts64.astype(np.float32), raster, grid, 2.2, 1.5,
                               seed=7)
    err = np.abs(out.reshape(want.shape).astype(np.float64) - want)
    assert float(np.abs(want).max()) > 1.0
    assert err.max() <= 1e-3, (err.max(), float(np.sqrt(np.mean(err ** 2))))
