"""GPU parity of crater shaping against the reference CPU path.

Inputs are what the reference hands its GPU backend (captured records, data and tile lists,
tests/golden/make_fixtures.py); the expected heights are the reference CPU path's for the same
scene. Tolerance: 1e-3 m absolute; the reference's own GPU test allows
2e-3 m (tests/unit/layers/craters/shaping/crater_kernel_test.cpp:212-272).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import grid_of
from terraingen_b200.layouts import CRATER_RECORD, CRATER_SHAPE_KERNEL

pytestmark = pytest.mark.gpu

SCENES = ["config1", "mpd", "complex", "diffused", "textured"]
TOLERANCE_M = 1e-3


def inputs(fx, name):
    kernel = fx[f"{name}_kernel"].view(CRATER_SHAPE_KERNEL)[0]
    records = fx[f"{name}_records"].view(CRATER_RECORD)
    data = fx[f"{name}_data"].view(np.float32)
    return kernel, records, data


@pytest.mark.parametrize("name", SCENES)
def test_craters_lists_form(device, crater_fixture, name):
    fx = crater_fixture
    kernel, records, data = inputs(fx, name)
    grid = grid_of(fx[f"{name}_grid"])
    heights = fx[f"{name}_heights"].view(np.float32).copy()
    lows_x = fx[f"{name}_x_lows"].view(np.float32)
    device.craters_apply_lists(kernel, records, data, fx[f"{name}_heads"].view(np.uint32),
                               fx[f"{name}_entries"].view(np.uint32),
                               fx[f"{name}_xs"].view(np.float32), lows_x,
                               fx[f"{name}_ys"].view(np.float32),
                               fx[f"{name}_y_lows"].view(np.float32), heights)
    expected = fx[f"{name}_expected"].reshape(-1)
    err = np.abs(heights.astype(np.float64) - expected)
    assert err.max() <= TOLERANCE_M, f"{name}: max {err.max():.3g} m"


@pytest.mark.parametrize("name", SCENES)
def test_craters_binned_form(device, crater_fixture, name):
    # The plain path: binning on the device from the records alone.
    fx = crater_fixture
    kernel, records, data = inputs(fx, name)
    grid = grid_of(fx[f"{name}_grid"])
    heights = np.zeros((grid.height, grid.width), np.float32)
    device.craters_apply(kernel, records, data, grid, heights)
    expected = fx[f"{name}_expected"]
    err = np.abs(heights.astype(np.float64) - expected)
    rms = float(np.sqrt(np.mean(err ** 2)))
    assert err.max() <= TOLERANCE_M, f"{name}: max {err.max():.3g} m, rms {rms:.3g}"


def test_binned_is_deterministic(device, crater_fixture):
    fx = crater_fixture
    kernel, records, data = inputs(fx, "config1")
    grid = grid_of(fx["config1_grid"])
    runs = []
    for _ in range(3):
        h = np.zeros((grid.height, grid.width), np.float32)
        device.craters_apply(kernel, records, data, grid, h)
        runs.append(h.view(np.uint32).copy())
    assert all(np.array_equal(runs[0], r) for r in runs[1:])


def test_binned_order_independent(device, crater_fixture):
    # Without datums craters add (apply_test.cpp:276-286): any record order gives the same bits.
    fx = crater_fixture
    kernel, records, data = inputs(fx, "config1")
    grid = grid_of(fx["config1_grid"])
    a = np.zeros((grid.height, grid.width), np.float32)
    device.craters_apply(kernel, records, data, grid, a)
    perm = np.random.default_rng(5).permutation(len(records))
    b = np.zeros_like(a)
    device.craters_apply(kernel, np.ascontiguousarray(records[perm]), data, grid, b)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_binned_tiles_independent(device, crater_fixture):
    # Evaluating a grid as four sub-grids gives the same heights as the whole.
    from terraingen_b200 import GridSpec

    fx = crater_fixture
    kernel, records, data = inputs(fx, "mpd")
    grid = grid_of(fx["mpd_grid"])
    whole = np.zeros((grid.height, grid.width), np.float32)
    device.craters_apply(kernel, records, data, grid, whole)
    hw, hh = grid.width // 2, grid.height // 2
    for (c0, r0, w, h) in [(0, 0, hw, hh), (hw, 0, grid.width - hw, hh),
                           (0, hh, hw, grid.height - hh), (hw, hh, grid.width - hw, grid.height - hh)]:
        sub = GridSpec(w, h, grid.x0 + c0 * grid.pixel, grid.y0 - r0 * grid.pixel, grid.pixel)
        part = np.zeros((h, w), np.float32)
        device.craters_apply(kernel, records, data, sub, part)
        # Tile membership differs at sub-grid edges only where a crater's reach ends mid-tile,
        # where it adds nothing; the heights agree to float rounding.
        assert np.abs(part - whole[r0:r0 + h, c0:c0 + w]).max() <= 1e-5


def test_nodata_cells_untouched(device, crater_fixture):
    fx = crater_fixture
    kernel, records, data = inputs(fx, "config1")
    grid = grid_of(fx["config1_grid"])
    h = np.zeros((grid.height, grid.width), np.float32)
    h[100:110, 100:110] = np.nan
    device.craters_apply(kernel, records, data, grid, h, nodata=(1, 0.0))
    assert np.all(np.isnan(h[100:110, 100:110]))
    assert np.isfinite(h[:100]).all()


def test_empty_inputs(device, crater_fixture):
    from terraingen_b200 import GridSpec

    fx = crater_fixture
    kernel, records, data = inputs(fx, "config1")
    h = np.zeros((0, 0), np.float32)
    device.craters_apply(kernel, records, data, GridSpec(0, 0, 0.0, 0.0, 1.0), h)
    grid = grid_of(fx["config1_grid"])
    h = np.full((grid.height, grid.width), 3.0, np.float32)
    device.craters_apply(kernel, records[:0], data, grid, h)
    assert np.all(h == 3.0)
    # A grid no crater reaches.
    far = GridSpec(64, 64, 1e5, 1e5, 1.0)
    h = np.full((64, 64), 1.0, np.float32)
    device.craters_apply(kernel, records, data, far, h)
    assert np.all(h == 1.0)


def test_datum_records_rejected_by_binned_form(device, crater_fixture):
    from terraingen_b200 import TgError

    fx = crater_fixture
    kernel, records, data = inputs(fx, "config1")
    grid = grid_of(fx["config1_grid"])
    rec = records.copy()
    rec["hasDatum"][0] = 1
    h = np.zeros((grid.height, grid.width), np.float32)
    with pytest.raises(TgError) as info:
        device.craters_apply(kernel, rec, data, grid, h)
    assert info.value.status == 3


def test_binned_odd_data_offsets_and_alignment(device, crater_fixture):
    # Record data may start at an odd float offset (the lean path reads harmonics as scalars);
    # device records that are not 16-byte aligned are refused, not read.
    import torch

    from terraingen_b200 import TgError

    fx = crater_fixture
    kernel, records, data = inputs(fx, "config1")
    grid = grid_of(fx["config1_grid"])
    base = np.zeros((grid.height, grid.width), np.float32)
    device.craters_apply(kernel, records, data, grid, base)
    shifted = records.copy()
    shifted["harmonicOffset"] += 1
    odd = np.zeros_like(base)
    device.craters_apply(kernel, shifted, np.concatenate([np.zeros(1, np.float32), data]), grid,
                         odd)
    assert np.array_equal(odd.view(np.uint32), base.view(np.uint32))
    raw = torch.zeros(records.nbytes + 16, dtype=torch.uint8, device="cuda")
    raw[8:8 + records.nbytes] = torch.from_numpy(records.view(np.uint8).copy()).cuda()
    h = torch.zeros((grid.height, grid.width), dtype=torch.float32, device="cuda")
    with pytest.raises(TgError):
        device.craters_apply(kernel, raw[8:8 + records.nbytes], torch.from_numpy(data).cuda(), grid,
                             h)


@pytest.mark.parametrize("name", ["config1", "complex"])
def test_staged_copy_timeout_is_reported_and_recovers(device, crater_fixture, name):
    # A wait limit of 0 polls makes the binned kernel (lean and general variants) give up on its
    # first staged copy at once, without a fault: TG_ERROR_TIMEOUT, then the same call with the
    # default limit gives the reference's heights.
    from terraingen_b200 import TgError

    fx = crater_fixture
    kernel, records, data = inputs(fx, name)
    grid = grid_of(fx[f"{name}_grid"])
    heights = np.zeros((grid.height, grid.width), np.float32)
    device.set_wait_limit(0)
    try:
        with pytest.raises(TgError) as error:
            device.craters_apply(kernel, records, data, grid, heights)
        assert error.value.status == 5  # TG_ERROR_TIMEOUT
    finally:
        device.set_wait_limit(1 << 26)
    heights = np.zeros((grid.height, grid.width), np.float32)
    device.craters_apply(kernel, records, data, grid, heights)
    err = np.abs(heights.astype(np.float64) - fx[f"{name}_expected"])
    assert err.max() <= TOLERANCE_M
