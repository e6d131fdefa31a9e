"""GPU tests of the batched form (tg_batch_*): many uneven tiles in one persistent launch.

- The source against the FP64 oracle (oracle/restate.cpp rs_fbm_grid_f64) at tiles near the
  origin and 1.7e6 m out, within 1e-4 m (the per-tile double lattice anchors keep float fractions).
- Craters and boulders against the plain per-tile path: the batch evaluates exactly the (cell,
  crater) and (cell, boulder) pairs the plain crater shaping and boulder bake evaluate on the
  batch's own source heights, and the heights agree within 1e-4 m.
- Kernel shapes (the autotuner's variants), replays and host/device memory give the same bits.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tiles():
    from terraingen_b200.workloads import uneven_tiles

    # Small tiles, denser craters and boulders than the benchmark's, half of them far out.
    return uneven_tiles(24, side=(40, 300), spacing=(0.25, 2.0), radius=1.7e6, density=1.0,
                        seed=5)


@pytest.fixture(scope="module")
def batch(device):
    from terraingen_b200.batch import Batch

    b = Batch(device)
    yield b
    b.close()


def _noise_only(ts):
    from dataclasses import replace

    from terraingen_b200.layouts import CRATER_RECORD

    tiles = ts.tiles.copy()
    for name in ("crater_begin", "crater_count", "data_begin", "boulder_begin", "boulder_count"):
        tiles[name] = 0
    return replace(ts, tiles=tiles, crater_records=np.zeros(0, CRATER_RECORD),
                   crater_data=np.zeros(0, np.float32), crater_footprints=np.zeros(0),
                   boulders=np.zeros((0, 5)))


def test_batch_source_matches_fp64_oracle(batch, tiles):
    ts = _noise_only(tiles)
    out = np.zeros(ts.output_floats, np.float32)
    batch.run(ts, out)
    rs = H.restate()
    f = ts.fractals[0]
    worst = 0.0
    far = 0
    for i, g in enumerate(ts.grids):
        want = np.zeros((g.height, g.width), np.float64)
        rs.rs_fbm_grid_f64(g.width, g.height, g.x0, g.y0, g.pixel, int(f["seed"]),
                           float(f["wavelength"]), float(f["amplitude"]), int(f["octaves"]),
                           float(f["lacunarity"]), float(f["gain"]), float(ts.elevation),
                           want.ctypes.data)
        got = ts.tile_view(out, i).astype(np.float64)
        err = np.abs(got - want).max()
        worst = max(worst, err)
        far += abs(g.x0) > 1e6 or abs(g.y0) > 1e6
    assert far >= 4, "the set must hold tiles at planetary distances"
    assert worst <= 1e-4, worst


def test_batch_matches_plain_path(device, batch, tiles):
    # The batch's source heights, then the plain path's craters and boulders per tile: the same
    # (cell, feature) pairs are evaluated, and heights agree to float rounding of the profiles
    # (the two kernels may contract multiply-adds differently; observed 3.5e-5 m at most).
    base = np.zeros(tiles.output_floats, np.float32)
    batch.run(_noise_only(tiles), base)
    out = np.zeros(tiles.output_floats, np.float32)
    batch.run(tiles, out)
    st = batch.stats()
    assert st["crater_pairs"] > 0 and st["boulder_pairs"] > 0
    shaped = 0
    pairs = {"crater_pairs": 0, "boulder_pairs": 0}
    worst = 0.0
    for i, g in enumerate(tiles.grids):
        t = tiles.tiles[i]
        h = np.ascontiguousarray(tiles.tile_view(base, i))
        r0, rn = int(t["crater_begin"]), int(t["crater_count"])
        d0 = int(t["data_begin"])
        d1 = int(tiles.tiles[i + 1]["data_begin"]) if i + 1 < len(tiles.grids) else len(
            tiles.crater_data)
        if rn:
            device.craters_apply(tiles.crater_kernel, tiles.crater_records[r0:r0 + rn],
                                 tiles.crater_data[d0:d1], g, h,
                                 footprints=tiles.crater_footprints[3 * r0:3 * (r0 + rn)])
            pairs["crater_pairs"] += device.counters()["crater_pairs"]
        b0, bn = int(t["boulder_begin"]), int(t["boulder_count"])
        if bn:
            device.boulders_bake(np.ascontiguousarray(tiles.boulders[b0:b0 + bn]), g, h,
                                 width=float(t["boulder_width"]))
            pairs["boulder_pairs"] += device.counters()["boulder_pairs"]
        got = tiles.tile_view(out, i)
        shaped += np.count_nonzero(got != tiles.tile_view(base, i))
        worst = max(worst, float(np.abs(got.astype(np.float64) - h).max()))
    assert st["crater_pairs"] == pairs["crater_pairs"], (st["crater_pairs"], pairs)
    assert st["boulder_pairs"] == pairs["boulder_pairs"], (st["boulder_pairs"], pairs)
    assert worst <= 1e-4, worst
    assert shaped > 1000


def test_batch_variants_replays_and_memory_agree(batch, tiles):
    import torch

    from terraingen_b200.batch import Batch

    batch.load(tiles)
    first = np.zeros(tiles.output_floats, np.float32)
    batch.evaluate(first)
    for v in range(len(Batch.variants())):
        batch.set_variant(v)
        out = np.zeros(tiles.output_floats, np.float32)
        batch.evaluate(out)
        batch.evaluate(out)  # a replay of the captured graph
        assert np.array_equal(out.view(np.uint32), first.view(np.uint32)), v
    before = batch.stats()
    dev = torch.zeros(tiles.output_floats, dtype=torch.float32, device="cuda")
    batch.evaluate(dev)
    batch.evaluate(dev)
    after = batch.stats()
    assert after["captures"] == before["captures"], "a replay must not re-capture"
    assert after["replays"] == before["replays"] + 2
    got = dev.cpu().numpy()
    for i in range(len(tiles.grids)):
        assert np.array_equal(tiles.tile_view(got, i), tiles.tile_view(first, i))


def test_batch_tune_picks_a_variant(batch, tiles):
    batch.load(tiles)
    ms = batch.tune(trials=2)
    st = batch.stats()
    assert np.isfinite(ms[st["variant"]])
    assert ms[st["variant"]] == min(m for m in ms if np.isfinite(m))


def test_batch_refuses_what_it_cannot_do(device, batch, tiles):
    from dataclasses import replace

    from terraingen_b200 import TgError

    # A crater datum needs the ordered drop-in form.
    rec = tiles.crater_records.copy()
    rec["hasDatum"][0] = 1
    with pytest.raises(TgError):
        batch.load(replace(tiles, crater_records=rec))
    # Features outside the batch's arrays.
    t = tiles.tiles.copy()
    t["crater_count"][1] = len(tiles.crater_records) + 1
    with pytest.raises(TgError):
        batch.load(replace(tiles, tiles=t))
    # An output too small.
    batch.load(tiles)
    with pytest.raises(TgError):
        batch.evaluate(np.zeros(tiles.output_floats - 1, np.float32))


def test_batch_empty_and_ragged(batch):
    from terraingen_b200.workloads import uneven_tiles

    ts = uneven_tiles(3, side=(1, 17), spacing=(0.5, 0.5), radius=10.0, density=1.0, seed=2)
    out = np.full(ts.output_floats, np.nan, np.float32)
    batch.run(ts, out)
    for i in range(3):
        assert np.isfinite(ts.tile_view(out, i)).all()
    empty = uneven_tiles(0)
    batch.run(empty, np.zeros(1, np.float32))


def test_batch_odd_data_offsets(batch, tiles):
    # Tiles whose data starts at an odd float offset (a tile before them with odd-length data):
    # the same heights as with even offsets.
    from dataclasses import replace

    even = np.zeros(tiles.output_floats, np.float32)
    batch.run(tiles, even)
    t = tiles.tiles.copy()
    t["data_begin"] += 1
    shifted = replace(tiles, tiles=t, crater_data=np.concatenate(
        [np.zeros(1, np.float32), tiles.crater_data]))
    odd = np.zeros(tiles.output_floats, np.float32)
    batch.run(shifted, odd)
    assert np.array_equal(odd.view(np.uint32), even.view(np.uint32))


def _with_points(ts, picks, per_tile, seed=0):
    """`ts` plus one point set per picked tile: `per_tile` of the tile's cell centers, naming the
    tile's own craters and boulders (the same records as the tile)."""
    from dataclasses import replace

    from terraingen_b200.batch import POINT_SET

    rng = np.random.default_rng(seed)
    sets = np.zeros(len(picks), POINT_SET)
    points, cells = [], []
    base = ts.output_floats
    for k, i in enumerate(picks):
        g, t = ts.grids[i], ts.tiles[i]
        n = min(per_tile, g.cells)
        flat = rng.choice(g.cells, n, replace=False)
        r, c = flat // g.width, flat % g.width
        points.append(np.stack([g.x0 + (c + 0.5) * g.pixel, g.y0 - (r + 0.5) * g.pixel], axis=1))
        cells.append((i, r, c))
        sets[k]["point_begin"] = sum(len(p) for p in points[:-1])
        sets[k]["point_count"] = n
        sets[k]["height_offset"] = base
        for name in ("crater_begin", "crater_count", "data_begin", "boulder_begin",
                     "boulder_count", "boulder_width"):
            sets[k][name] = t[name]
        base += n
    return replace(ts, point_sets=sets, points=np.concatenate(points)), cells


def test_batch_point_sets_match_tiles(batch, tiles):
    # Points at cell centers of three tiles (one far out), sharing the tiles' records: heights
    # within 1e-4 m of the tiles' cells.
    far = max(range(len(tiles.grids)), key=lambda i: abs(tiles.grids[i].x0) + abs(tiles.grids[i].y0))
    ts, cells = _with_points(tiles, [0, 3, far], 2000)
    out = np.zeros(ts.output_floats, np.float32)
    batch.run(ts, out)
    assert batch.stats()["crater_pairs"] > 0
    for k, (i, r, c) in enumerate(cells):
        got = ts.point_view(out, k).astype(np.float64)
        want = ts.tile_view(out, i)[r, c].astype(np.float64)
        assert np.abs(got - want).max() <= 1e-4, (k, np.abs(got - want).max())


def test_batch_points_source_matches_fp64_oracle(batch, tiles):
    ts, _ = _with_points(_noise_only(tiles), [1, 2], 500, seed=4)
    pts = ts.points.copy()
    pts[:500] += 1.6e6  # far out, where float positions lose the lattice fraction
    from dataclasses import replace

    ts = replace(ts, points=pts)
    out = np.zeros(ts.output_floats, np.float32)
    batch.run(ts, out)
    rs = H.restate()
    f = ts.fractals[0]
    for k in range(2):
        p = ts.point_sets[k]
        xy = ts.points[int(p["point_begin"]):int(p["point_begin"]) + int(p["point_count"])]
        want = np.array([ts.elevation + rs.rs_fbm2_f64(x, y, int(f["seed"]), float(f["wavelength"]),
                                                       float(f["amplitude"]), int(f["octaves"]),
                                                       float(f["lacunarity"]), float(f["gain"]))
                         for x, y in xy])
        got = ts.point_view(out, k).astype(np.float64)
        assert np.abs(got - want).max() <= 1e-4, (k, np.abs(got - want).max())


def test_batch_shared_records(batch, tiles):
    # Two tiles over the same grid naming the same records and boulders: the same heights.
    from dataclasses import replace

    t = np.concatenate([tiles.tiles, tiles.tiles[:1]])
    t["height_offset"][-1] = tiles.output_floats
    ts = replace(tiles, tiles=t, grids=tiles.grids + tiles.grids[:1])
    out = np.zeros(ts.output_floats, np.float32)
    batch.run(ts, out)
    a = ts.tile_view(out, 0)
    b = ts.tile_view(out, len(t) - 1)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_batch_pinned_host_output_equals_device(device, tiles):
    # Page-locked host heights cross chunk by chunk while later chunks are evaluated: the same
    # bits as a device evaluation, on a fresh batch (whose first run grows its bins' entries and
    # runs again whole) and on the replays after it.
    import torch

    from terraingen_b200.batch import Batch

    dev = torch.zeros(tiles.output_floats, dtype=torch.float32, device="cuda")
    with Batch(device) as fresh:
        fresh.load(tiles)
        pinned = torch.zeros(tiles.output_floats, dtype=torch.float32).pin_memory().numpy()
        fresh.evaluate(pinned)
        fresh.evaluate(dev)
        want = dev.cpu().numpy()
        for i in range(len(tiles.grids)):
            assert np.array_equal(tiles.tile_view(pinned, i), tiles.tile_view(want, i)), i
        pinned[:] = np.nan
        fresh.evaluate(pinned)
        fresh.evaluate(pinned)
        for i in range(len(tiles.grids)):
            assert np.array_equal(tiles.tile_view(pinned, i), tiles.tile_view(want, i)), i
