"""GPU tests of the served form (tg_server_*): continuous batching of tile and point requests.

- A request's heights are the same alone (on a fresh server) and in a mix of requests.
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

    opts = dem_stack_options(slots=1)
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

    opts = dem_stack_options(slots=1)
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
        dev = run_stream(s, reqs, realtime=False, keep=True, device=True)
    for r in reqs:
        a = host.outputs[r.rid]
        b = dev.outputs[r.rid].cpu().numpy()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), r.kind


def test_served_points_equal_batched_points(device):
    # Points read their regions' resident cell lists; the batch engine bins the same points
    # against tg_crater_batch's records over their bounding box: the same heights.
    from terraingen_b200.batch import POINT_SET, Batch, TileSet
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options
    from terraingen_b200.workloads import crater_batch

    opts = dem_stack_options(slots=1)
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
