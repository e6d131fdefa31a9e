"""Host-side checks of the batched form: the tile layout the C ABI reads, the output layout, and
the uneven-tile workload's shape (sides, spacings, distances, per-tile ranges)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from terraingen_b200 import _native as N
from terraingen_b200.batch import TILE, layout
from terraingen_b200.device import centered
from terraingen_b200.workloads import uneven_tiles


def test_tile_layout_matches_the_header():
    assert TILE.itemsize == C.sizeof(N.Tile) == 96
    for name, _ in N.Tile._fields_:
        if name == "grid":
            continue
        assert TILE.fields[name][1] == getattr(N.Tile, name).offset, name
    assert C.sizeof(N.BatchInput) == 128
    from terraingen_b200.batch import POINT_SET

    assert POINT_SET.itemsize == C.sizeof(N.PointSet) == 48
    assert C.sizeof(N.BatchStats) == 88


def test_output_layout_is_aligned_and_disjoint():
    grids = [centered(65, 70, 1.0), centered(1, 1, 0.5), centered(1025, 3, 2.0)]
    offsets, pitch = layout(grids)
    assert list(pitch) == [68, 4, 1028]
    assert all(int(o) % 4 == 0 for o in offsets)
    ends = [int(o) + int(p) * g.height for o, p, g in zip(offsets, pitch, grids)]
    assert ends[:-1] == [int(o) for o in offsets[1:]]


def test_uneven_tiles_shape():
    ts = uneven_tiles(40, seed=3)
    t = ts.tiles
    assert ((t["width"] >= 65) & (t["width"] <= 1025)).all()
    assert (t["width"] == t["height"]).all()
    pixel = t["pixel_width"]
    assert ((pixel >= 0.25) & (pixel <= 2.0)).all()
    cx = t["origin_x"] + 0.5 * t["width"] * pixel
    cy = t["origin_y"] - 0.5 * t["height"] * pixel
    assert (np.hypot(cx, cy) <= 1.7e6 + 1.0).all()
    # Records, data and boulders lie tile after tile.
    assert t["crater_begin"][0] == 0 and t["boulder_begin"][0] == 0
    assert (t["crater_begin"][1:] == t["crater_begin"][:-1] + t["crater_count"][:-1]).all()
    assert (t["boulder_begin"][1:] == t["boulder_begin"][:-1] + t["boulder_count"][:-1]).all()
    assert (np.diff(t["data_begin"].astype(np.int64)) >= 0).all()
    assert int(t["crater_begin"][-1] + t["crater_count"][-1]) == len(ts.crater_records)
    assert len(ts.crater_footprints) == 3 * len(ts.crater_records)
    # The same seed gives the same batch.
    again = uneven_tiles(40, seed=3)
    assert np.array_equal(again.tiles, ts.tiles)
    assert np.array_equal(again.crater_records, ts.crater_records)
    assert ts.output_floats == int((t["height_offset"] + (t["height"].astype(np.int64) - 1) *
                                    t["pitch"] + t["width"]).max())
