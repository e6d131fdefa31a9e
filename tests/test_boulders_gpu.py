"""GPU parity of boulder baking against the reference CPU path: the boulders the reference's
BoulderLayer draws, baked on the heights beneath them, against the reference heights with them.
Tolerance 1e-3 m (the dome math is FP64 in both; only asin/sqrt rounding may differ)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, grid_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN / "boulders.npz"))


@pytest.mark.parametrize("name", ["dense", "fine"])
def test_boulders_match_reference(device, fx, name):
    grid = grid_of(fx[f"{name}_grid"])
    boulders = np.ascontiguousarray(fx[f"{name}_boulders"])
    heights = fx[f"{name}_base"].copy()
    device.boulders_bake(boulders, grid, heights, width=grid.pixel)
    err = np.abs(heights.astype(np.float64) - fx[f"{name}_expected"])
    assert err.max() <= 1e-3, err.max()
    assert np.count_nonzero(heights != fx[f"{name}_base"]) > 1000


def test_boulders_order_free(device, fx):
    grid = grid_of(fx["dense_grid"])
    boulders = np.ascontiguousarray(fx["dense_boulders"])
    a = fx["dense_base"].copy()
    device.boulders_bake(boulders, grid, a, width=grid.pixel)
    b = fx["dense_base"].copy()
    perm = np.random.default_rng(3).permutation(len(boulders))
    device.boulders_bake(np.ascontiguousarray(boulders[perm]), grid, b, width=grid.pixel)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_boulders_point_dome_and_edges(device):
    # A zero width samples the dome at the point (DomeHeight, boulder_relief.cpp:44-50); a boulder
    # off the grid changes nothing; an invalid boulder is refused.
    from terraingen_b200 import TgError, centered

    grid = centered(16, 16, 1.0)
    h = np.zeros((16, 16), np.float32)
    one = np.array([[0.0, 0.0, 6.0, 2.0, 1.0]])
    device.boulders_bake(one, grid, h, width=0.0)
    cy, cx = np.mgrid[0:16, 0:16]
    x = -8.0 + cx + 0.5
    y = 8.0 - cy - 0.5
    r2 = (x * x + y * y) / 9.0
    want = np.where(r2 < 1.0, 2.0 * np.sqrt(np.clip(1.0 - r2, 0, None)), 0.0)
    assert np.abs(h - want).max() < 1e-6
    far = np.zeros((16, 16), np.float32)
    device.boulders_bake(np.array([[1e4, 1e4, 3.0, 1.0, 1.0]]), grid, far, width=1.0)
    assert not far.any()
    with pytest.raises(TgError):
        device.boulders_bake(np.array([[0.0, 0.0, -1.0, 1.0, 1.0]]), grid, far, width=1.0)


def test_staged_copy_timeout_is_reported_and_recovers(device, fx):
    # A wait limit of 0 polls makes every bin's first staged-copy wait give up at once (no fault:
    # the copies still land, and each CTA waits, bounded, for its copies in flight before it
    # leaves). The call reports TG_ERROR_TIMEOUT and the device keeps working: with the default
    # limit restored the same bake gives the reference's heights.
    from terraingen_b200 import TgError

    grid = grid_of(fx["dense_grid"])
    boulders = np.ascontiguousarray(fx["dense_boulders"])
    heights = fx["dense_base"].copy()
    device.set_wait_limit(0)
    try:
        with pytest.raises(TgError) as error:
            device.boulders_bake(boulders, grid, heights, width=grid.pixel)
        assert error.value.status == 5  # TG_ERROR_TIMEOUT
    finally:
        device.set_wait_limit(1 << 26)
    heights = fx["dense_base"].copy()
    device.boulders_bake(boulders, grid, heights, width=grid.pixel)
    assert np.abs(heights.astype(np.float64) - fx["dense_expected"]).max() <= 1e-3
