"""GPU parity of diamond-square refinement against the reference's DiamondSquareUpsampler, and
the Philox4x32-10 draws against the Random123 known answers the reference's tests use
(tests/unit/random/philox_test.cpp:14-23) and the restated oracle."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, grid_of

pytestmark = pytest.mark.gpu

# Heights are FP64 nodes read to float; the displacements' normals are a float Box-Muller on the
# exact uniforms (within 1e-5 of the double normal), so the heights stay far below the 1e-3 m of
# the configurations.
TOLERANCE_M = 1e-3


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLDEN / "ds.npz"))


@pytest.mark.parametrize("name", ["dem5m", "exact", "tenfold", "dem5m_cr", "tenfold_cr"])
def test_ds_matches_reference(device, fx, name):
    # Bilinear and Catmull-Rom (the _cr cases) refinements against the reference's.
    pg = grid_of(fx[f"{name}_post_grid"])
    grid = grid_of(fx[f"{name}_grid"])
    fd, scale, seed, interp = fx[f"{name}_options"]
    heights = np.zeros((grid.height, grid.width), np.float32)
    device.ds_refine(fx[f"{name}_posts"], pg, grid, heights, fd, scale, int(seed), int(interp))
    err = np.abs(heights.astype(np.float64) - fx[f"{name}_expected"])
    assert err.max() <= TOLERANCE_M, (name, err.max())


def test_philox_known_answers(device):
    sextets = np.array([[0, 0, 0, 0, 0, 0],
                        [0xffffffff] * 6,
                        [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344, 0xa4093822, 0x299f31d0]],
                       np.uint32)
    words, _ = device.philox_probe(sextets)
    assert [list(map(int, w)) for w in words] == [
        [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8],
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd],
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]]


def test_displacement_draws_match_oracle(device):
    from oracle import harness as H

    rs = H.restate()
    rng = np.random.default_rng(4)
    cols = rng.integers(-50000, 50000, 20000)
    rows = rng.integers(-50000, 50000, 20000)
    levels = rng.integers(1, 6, 20000)
    sext = np.zeros((20000, 6), np.uint32)
    sext[:, 0] = cols.astype(np.int64).astype(np.uint32)
    sext[:, 1] = rows.astype(np.int64).astype(np.uint32)
    sext[:, 2] = levels
    sext[:, 4] = 7
    sext[:, 5] = 0x524D4450
    words, normals = device.philox_probe(sext)
    want = np.array([rs.rs_ds_normal(int(cols[i]), int(rows[i]), int(levels[i]), 7)
                     for i in range(len(cols))])
    # Box-Muller in float on the exact uniforms: a few 1e-7 of the radius (at most 8.6), the
    # hardware cosine within 4e-7.
    err = np.abs(normals - want)
    assert err.max() <= 1e-5, (int(err.argmax()), float(err.max()))
    assert float(np.abs(want).max()) > 3.0


def test_ds_deterministic_and_windowed(device, fx):
    # A window of the output is the same as the window cut from the whole: node values do not
    # depend on the box they are computed in.
    from terraingen_b200 import GridSpec

    pg = grid_of(fx["exact_post_grid"])
    grid = grid_of(fx["exact_grid"])
    fd, scale, seed, _ = fx["exact_options"]
    whole = np.zeros((grid.height, grid.width), np.float32)
    device.ds_refine(fx["exact_posts"], pg, grid, whole, fd, scale, int(seed))
    again = np.zeros_like(whole)
    device.ds_refine(fx["exact_posts"], pg, grid, again, fd, scale, int(seed))
    assert np.array_equal(whole.view(np.uint32), again.view(np.uint32))
    c0, r0, w, h = 37, 51, 90, 70
    sub = GridSpec(w, h, grid.x0 + c0 * grid.pixel, grid.y0 - r0 * grid.pixel, grid.pixel)
    part = np.zeros((h, w), np.float32)
    device.ds_refine(fx["exact_posts"], pg, sub, part, fd, scale, int(seed))
    assert np.array_equal(part.view(np.uint32), whole[r0:r0 + h, c0:c0 + w].view(np.uint32))


def test_ds_zero_scale_is_interpolation(device, fx):
    # With no displacement, refinement averages: the result stays within the posts' range.
    pg = grid_of(fx["dem5m_post_grid"])
    grid = grid_of(fx["dem5m_grid"])
    posts = fx["dem5m_posts"]
    heights = np.zeros((grid.height, grid.width), np.float32)
    device.ds_refine(posts, pg, grid, heights, 2.2, 0.0, 1)
    assert heights.min() >= posts.min() - 1e-3 and heights.max() <= posts.max() + 1e-3


@pytest.mark.parametrize("name", ["dem5m", "exact", "tenfold", "tenfold_cr"])
def test_ds_window_of_posts_matches_whole(device, fx, name):
    # A 64^2 block inside the fixture's grid, refined from only the posts over its bounds and
    # eight posts around (tg_ds_refine_window: the node frame still the whole lattice's), is the
    # whole lattice's refinement of that block bit for bit.
    import math

    from terraingen_b200 import GridSpec

    pg = grid_of(fx[f"{name}_post_grid"])
    grid = grid_of(fx[f"{name}_grid"])
    fd, scale, seed, interp = fx[f"{name}_options"]
    interp = int(interp)
    posts = fx[f"{name}_posts"]
    block = GridSpec(64, 64, grid.x0 + 100 * grid.pixel, grid.y0 - 90 * grid.pixel, grid.pixel)
    whole = np.zeros((64, 64), np.float32)
    device.ds_refine(posts, pg, block, whole, fd, scale, int(seed), interp)
    c0 = max(0, math.floor((block.x0 - pg.x0) / pg.pixel) - 8)
    c1 = min(pg.width, math.ceil((block.x0 + 64 * block.pixel - pg.x0) / pg.pixel) + 8)
    r0 = max(0, math.floor((pg.y0 - block.y0) / pg.pixel) - 8)
    r1 = min(pg.height, math.ceil((pg.y0 - block.y0 + 64 * block.pixel) / pg.pixel) + 8)
    assert c0 > 0 and r0 > 0 and c1 < pg.width and r1 < pg.height
    window = np.ascontiguousarray(posts[r0:r1, c0:c1])
    part = np.zeros_like(whole)
    device.ds_refine(window, pg, block, part, fd, scale, int(seed), interp, window=(c0, r0))
    assert np.array_equal(part.view(np.uint32), whole.view(np.uint32)), name
    # The same posts passed as a lattice of their own draw other displacements.
    alone = np.zeros_like(whole)
    shifted = GridSpec(c1 - c0, r1 - r0, pg.x0 + c0 * pg.pixel, pg.y0 - r0 * pg.pixel, pg.pixel)
    device.ds_refine(window, shifted, block, alone, fd, scale, int(seed), interp)
    assert not np.array_equal(alone, whole)
