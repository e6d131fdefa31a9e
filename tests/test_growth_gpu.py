"""The layers' binning sizes itself on the device: the entries get the capacity the device already
holds, the kernels after the scan do nothing when the scan's total is larger, and the call grows
the entries and runs the layers again before it returns. A fresh device (empty slots) given a
few craters and boulders that each cover most bins of a grid takes that path on its first call;
its heights and pair counts must be those of the second call, which fits at once."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs():
    from terraingen_b200 import workloads as W
    from terraingen_b200.device import centered

    grid = centered(2048, 2048, 1.0)
    # Few large craters (300-500 m): each covers hundreds to thousands of 32 x 32 bins, far past
    # a first guess of four entries a crater plus one a bin.
    population = W.crater_population(5, 1.7, 300.0, 500.0)
    craters = W.crater_batch(population, grid, shaping=W.config2_shaping())
    # Thirteen boulders whose domes cover the whole grid: 13 x 4096 entries.
    stones = np.zeros((13, 5), np.float64)
    stones[:, 0] = np.linspace(-10.0, 10.0, 13)
    stones[:, 2] = 2500.0
    stones[:, 3] = 1.0
    stones[:, 4] = 1.0
    fr = np.array([W.fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)])
    return grid, craters, stones, fr


def test_evaluate_grows_entries_on_a_fresh_device():
    from terraingen_b200 import Device

    grid, craters, stones, fr = _inputs()
    assert 20 <= len(craters[1]) <= 400
    with Device() as fresh:
        first = np.zeros((grid.height, grid.width), np.float32)
        fresh.evaluate(grid, first, fractals=fr, craters=craters, boulders=stones,
                       boulder_width=grid.pixel)
        pairs_first = fresh.counters()
        again = np.zeros_like(first)
        fresh.evaluate(grid, again, fractals=fr, craters=craters, boulders=stones,
                       boulder_width=grid.pixel)
        assert fresh.counters() == pairs_first
    assert np.array_equal(first.view(np.uint32), again.view(np.uint32))
    assert pairs_first["crater_pairs"] > 0 and pairs_first["boulder_pairs"] > 0


def test_layer_calls_grow_entries_on_a_fresh_device():
    import torch

    from terraingen_b200 import Device

    grid, craters, stones, fr = _inputs()
    kernel, records, data, foot = craters
    with Device() as warm:
        base = np.zeros((grid.height, grid.width), np.float32)
        warm.noise_source(fr, grid, base)
        # Calls that grow the device's entries, then the ones that fit at once.
        scratch = base.copy()
        warm.craters_apply(kernel, records, data, grid, scratch, footprints=foot)
        warm.boulders_bake(stones, grid, scratch, width=grid.pixel)
        want = base.copy()
        warm.craters_apply(kernel, records, data, grid, want, footprints=foot)
        warm.boulders_bake(stones, grid, want, width=grid.pixel)
    for memory in ("host", "device"):
        with Device() as fresh:
            got = base.copy()
            if memory == "device":
                dev = torch.from_numpy(got).cuda()
                rec_t = torch.from_numpy(records.view(np.uint8).copy()).cuda()
                fresh.craters_apply(kernel, rec_t, torch.from_numpy(data).cuda(), grid, dev,
                                    footprints=torch.from_numpy(foot).cuda())
                fresh.boulders_bake(torch.from_numpy(stones).cuda(), grid, dev,
                                    width=grid.pixel)
                got = dev.cpu().numpy()
            else:
                fresh.craters_apply(kernel, records, data, grid, got, footprints=foot)
                fresh.boulders_bake(stones, grid, got, width=grid.pixel)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), memory
