"""The benchmark's terrain, built by the product alone (tg_crater_batch, tg_boulder_generate,
tg_evaluate), against the reference CPU path evaluating the same scene (oracle/_ref).

A 385^2 window of the 4097^2 terrain at 0.5 m: the fBm source, 200,000 craters per tile area and
the boulders of 1,000,000 per tile area, within 1e-3 m of the reference's heights everywhere.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import harness as H

pytestmark = pytest.mark.gpu


def test_terrain_window_matches_reference(device):
    from terraingen_b200.workloads import terrain4097, terrain4097_reference_scene

    side = 385
    w = terrain4097(side, 0.5)
    assert len(w.crater_records) > 1000 and len(w.boulders) > 50
    got = np.zeros((side, side), np.float32)
    device.evaluate(w.grid, got, fractals=w.fractals, elevation=w.elevation,
                    craters=(w.crater_kernel, w.crater_records, w.crater_data,
                             w.crater_footprints),
                    boulders=w.boulders, boulder_width=w.boulder_width)
    grid, fr, craters, boulders = terrain4097_reference_scene(side, 0.5)
    assert grid == w.grid
    scene = H.make_scene(grid, source_fractals=fr, craters=craters, boulders=boulders)
    assert np.array_equal(H.boulders(H.reference(), scene).view(np.uint64),
                          w.boulders.view(np.uint64))
    want, _ = H.evaluate(H.reference(), scene, 0, 0)
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= 1e-3, (err.max(), float(np.sqrt(np.mean(err ** 2))))
