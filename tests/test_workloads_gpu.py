"""The benchmark's terrain, built by the product alone (tg_crater_batch, tg_boulder_generate,
tg_evaluate), against the reference CPU path evaluating the same scene (oracle/_ref).

Windows of the 4097^2 terrain at 0.5 m: the fBm source, 200,000 craters per tile area with the
configuration's central peaks and terraces mapped onto the reference's options (complex craters
from 4.47 m, every one with massif peaks; terraces from 200 m; terraingen_b200.workloads), and the
boulders of 1,000,000 per tile area, within 1e-3 m of the reference's heights everywhere. A
scene with many terraced and peaked craters checks the binned kernel's two queues (lean entries,
complex ones included, and heavy entries such as terraces) against the reference.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import harness as H

pytestmark = pytest.mark.gpu

TOLERANCE_M = 1e-3


@pytest.mark.parametrize("cx,cy", [(0.0, 0.0), (-700.0, 820.0)])
def test_terrain_window_matches_reference(device, cx, cy):
    from terraingen_b200.device import centered
    from terraingen_b200.workloads import terrain4097, terrain4097_reference_scene

    side = 385
    w = terrain4097(side, 0.5, cx, cy)
    assert len(w.crater_records) > 1000 and len(w.boulders) > 50
    assert np.count_nonzero(w.crater_records["peakCount"]) > 20
    got = np.zeros((side, side), np.float32)
    device.evaluate(w.grid, got, fractals=w.fractals, elevation=w.elevation,
                    craters=(w.crater_kernel, w.crater_records, w.crater_data,
                             w.crater_footprints),
                    boulders=w.boulders, boulder_width=w.boulder_width)
    _, fr, craters, boulders = terrain4097_reference_scene(side, 0.5)
    grid = centered(side, side, 0.5, cx, cy)
    assert grid == w.grid
    scene = H.make_scene(grid, source_fractals=fr, craters=craters, boulders=boulders)
    assert np.array_equal(H.boulders(H.reference(), scene).view(np.uint64),
                          w.boulders.view(np.uint64))
    want, _ = H.evaluate(H.reference(), scene, 0, 0)
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= TOLERANCE_M, (err.max(), float(np.sqrt(np.mean(err ** 2))))


def test_terraced_peaked_scene_matches_reference(device):
    # Complex craters over Fassett-Thomson from 60 m with the default apply: massif peaks (lean
    # queue) and wall terraces from 80 m (heavy queue) in the same binned launch.
    from terraingen_b200 import _native as N
    from terraingen_b200.device import centered
    from terraingen_b200.workloads import crater_batch

    grid = centered(192, 192, 2.0)
    fields = dict(seed=9, sfdCoefficient=0.6, minDiameter=8.0, maxDiameter=300.0, profile=2,
                  transitionDiameter=60.0, terraceOnset=80.0, terraceFull=200.0)
    pop = N.Population(seed=9, sfd_coefficient=0.6, sfd_exponent=2.0, min_diameter=8.0,
                       max_diameter=300.0, lifetime_gyr=1.0, depth_ratio=0.2, rim_ratio=0.04,
                       cutoff_depth_ratio=0.04, cell_size_factor=16.0, margin_radii=0.0,
                       min_resolved_diameter=0.0)
    shaping = N.Shaping(profile=2, irregular=1, transition_diameter=60.0, terrace_onset=80.0,
                        terrace_full=200.0, terrace_min_freshness=0.3)
    kernel, records, data, foot = crater_batch(pop, grid, shaping=shaping)
    assert np.count_nonzero(records["terraceCount"]) > 0
    assert np.count_nonzero(records["peakCount"]) > 0
    got = np.zeros((grid.height, grid.width), np.float32)
    device.craters_apply(kernel, records, data, grid, got, footprints=foot)
    want, _ = H.evaluate(H.reference(), H.make_scene(grid, craters=fields), 0, 0)
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= TOLERANCE_M, (err.max(), float(np.sqrt(np.mean(err ** 2))))
