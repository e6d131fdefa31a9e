"""GPU tests of point queries against the reference's own point path: Terrain::HeightsAt, which
runs EvaluatePoints (src/pipeline/terrain.cpp:133-154: points in Morton-ordered batches, each
batch's crater and boulder layers prepared over its own area) on the reference CPU build.

- Batched point sets (tg_batch) on the synthetic terrain's stack (fBm, craters with the peak and
  terrace mapping, boulders) at scattered positions within 1e-3 m.
- Served point queries (tg_server) on the fBm-at-every-cell stack within 1e-3 m.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import harness as H

pytestmark = pytest.mark.gpu

TOLERANCE_M = 1e-3


def _scatter(grid, n, seed):
    """n points uniformly inside `grid`'s extent, one cell in from its edges."""
    rng = np.random.default_rng(seed)
    span_x = (grid.width - 2) * grid.pixel
    span_y = (grid.height - 2) * grid.pixel
    return np.stack([grid.x0 + grid.pixel + span_x * rng.random(n),
                     grid.y0 - grid.pixel - span_y * rng.random(n)], axis=1)


def test_batched_points_match_reference_points(device):
    from terraingen_b200.batch import POINT_SET, TILE, Batch, TileSet
    from terraingen_b200.workloads import terrain4097, terrain4097_reference_scene

    w = terrain4097(385, 0.5, 310.0, -205.0)
    xy = _scatter(w.grid, 4000, 3)
    sets = np.zeros(1, POINT_SET)
    sets["point_count"] = len(xy)
    sets["crater_count"] = len(w.crater_records)
    sets["boulder_count"] = len(w.boulders)
    sets["boulder_width"] = w.boulder_width
    ts = TileSet(tiles=np.zeros(0, TILE), fractals=w.fractals, elevation=w.elevation,
                 crater_kernel=w.crater_kernel, crater_records=w.crater_records,
                 crater_data=w.crater_data, crater_footprints=w.crater_footprints,
                 boulders=w.boulders, point_sets=sets, points=xy)
    got = np.zeros(ts.output_floats, np.float32)
    with Batch(device) as b:
        b.run(ts, got)
        stats = b.stats()
    assert stats["crater_pairs"] > 1000 and stats["boulder_pairs"] > 0
    _, fr, craters, boulders = terrain4097_reference_scene(385, 0.5)
    scene = H.make_scene(w.grid, source_fractals=fr, craters=craters, boulders=boulders)
    want = H.points(H.reference(), scene, xy, w.boulder_width)
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= TOLERANCE_M, (err.max(), float(np.sqrt(np.mean(err ** 2))))


def test_served_points_match_reference_points(device):
    from terraingen_b200.device import GridSpec
    from terraingen_b200.serve import Server, dem_stack_options

    opts = dem_stack_options(slots=1, refine=False)
    box = GridSpec(1200, 1200, 150.0, 20.0, opts.point_spacing)
    xy = _scatter(box, 3000, 5)
    got = np.empty(len(xy), np.float32)
    with Server(device, opts) as s:
        s.submit_points(1, xy, got)
        assert s.drain() == [1]
    p = opts.craters
    craters = dict(seed=p.seed, sfdCoefficient=p.sfd_coefficient, sfdExponent=p.sfd_exponent,
                   minDiameter=p.min_diameter, maxDiameter=p.max_diameter,
                   lifetimeGyr=p.lifetime_gyr, depthRatio=p.depth_ratio, rimRatio=p.rim_ratio,
                   profile=0)
    scene = H.make_scene(box, source_fractals=opts._fractals, craters=craters)
    want = H.points(H.reference(), scene, xy, opts.point_spacing)
    # The craters reach the points: the heights are not the source alone.
    source = H.points(H.reference(), H.make_scene(box, source_fractals=opts._fractals), xy,
                      opts.point_spacing)
    assert np.count_nonzero(np.abs(want - source) > 0.01) > 100
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= TOLERANCE_M, (err.max(), float(np.sqrt(np.mean(err ** 2))))
