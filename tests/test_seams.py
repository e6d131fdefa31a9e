"""The seam restatement (oracle/seams.py) against the reference's own seams (tests/golden/seams.npz).

Two scenes (a hole inside a 1 m patch; one of 2 x 2 patches at 2 m whose gap reaches the raster's
edges), each joined by Feather, Height and Slope:
  - the lattice samples are the rasters' own values on the lattice's inner posts (the lattice
    is the rasters' grid padded by ceil(reach / spacing) + 3 posts) and no data on the pad;
  - Feather's field is bit-exact (the chamfer distances and carried values in float);
  - Height / Slope, solved directly, are within 1e-6 m of the reference's multigrid-
    preconditioned conjugate gradients;
  - reading the field between posts and filling the gaps (FillGridGaps) gives the chain's
    heights bit for bit, on the rasters' grid and on a grid of half the spacing.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN, grid_of
from oracle import seams as S

CASES = [(scene, mode) for scene in ("hole", "patch") for mode in ("feather", "height", "slope")]


@pytest.fixture(scope="module")
def z():
    return dict(np.load(GOLDEN / "seams.npz"))


def _spacing(z, key):
    lat = z[f"{key}_lattice"]
    return float(lat[3]), float(-lat[7])


@pytest.mark.parametrize("scene,mode", CASES)
def test_lattice_samples_are_the_rasters(z, scene, mode):
    key = f"{scene}_{mode}"
    earlier, later = z[f"{scene}_earlier"], z[f"{scene}_later"]
    _, width, decay = z[f"{key}_options"]
    g = grid_of(z[f"{scene}_grid"])
    reach = width if mode == "feather" else 3.0 * decay
    pad = math.ceil(reach / g.pixel) + 3
    lat = z[f"{key}_lattice"]
    assert (int(lat[0]), int(lat[1])) == (g.width + 2 * pad, g.height + 2 * pad)
    assert lat[2] == g.x0 - pad * g.pixel and lat[5] == g.y0 + pad * g.pixel
    data, diff = z[f"{key}_data"], z[f"{key}_difference"]
    inner = (slice(pad, pad + g.height), slice(pad, pad + g.width))
    assert np.array_equal(data[inner], (~np.isnan(earlier)).astype(np.uint8))
    want = (earlier.astype(np.float64) - later).astype(np.float32)
    assert np.array_equal(np.isnan(diff[inner]), np.isnan(want))
    assert np.array_equal(diff[inner][~np.isnan(want)], want[~np.isnan(want)])
    outer = np.ones(data.shape, bool)
    outer[inner] = False
    assert not data[outer].any() and np.isnan(diff[outer]).all()


@pytest.mark.parametrize("scene", ["hole", "patch"])
def test_feather_restatement_is_bit_exact(z, scene):
    key = f"{scene}_feather"
    dx, dy = _spacing(z, key)
    got = S.feather(z[f"{key}_data"], z[f"{key}_difference"], dx, dy, float(z[f"{key}_options"][1]))
    want = z[f"{key}_field"]
    assert np.count_nonzero(want) > 1000
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("scene,mode", [(s, m) for s in ("hole", "patch") for m in ("height",
                                                                                    "slope")])
def test_screened_solve_restatement(z, scene, mode):
    key = f"{scene}_{mode}"
    dx, dy = _spacing(z, key)
    got = S.solve(z[f"{key}_data"], z[f"{key}_difference"], dx, dy, mode,
                  float(z[f"{key}_options"][2]))
    want = z[f"{key}_field"]
    assert np.abs(want).max() > 1.0
    err = np.abs(got.astype(np.float64) - want).max()
    assert err <= 1e-6, err


@pytest.mark.parametrize("scene,mode", CASES)
def test_fill_restatement_is_the_chain(z, scene, mode):
    key = f"{scene}_{mode}"
    lattice = tuple(z[f"{key}_lattice"][2:])
    for prefix, grid in (("", z[f"{scene}_grid"]), ("fine_", z[f"{scene}_fine_grid"])):
        heights = z[f"{scene}_{prefix}earlier"]
        got = S.fill(z[f"{key}_field"], lattice, z[f"{scene}_{prefix}later"], grid_of(grid),
                     heights)
        want = z[f"{key}_{prefix}chain"]
        assert np.isnan(heights).sum() > 500
        assert np.count_nonzero(got != z[f"{scene}_{prefix}later"]) > 0
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), prefix


def test_distances_carry_the_nearest_difference():
    # A single post with data: distances are the chamfer metric, and every post carries its value.
    data = np.zeros((9, 11), np.uint8)
    data[4, 5] = 1
    values = np.zeros((9, 11), np.float32)
    values[4, 5] = 2.5
    d, carried = S.distances(data, 1.0, 2.0, values)
    diag = np.float32(math.hypot(1.0, 2.0))
    assert d[4, 5] == 0.0 and d[4, 8] == 3.0 and d[2, 5] == 4.0 and d[3, 6] == diag
    assert (carried == 2.5).all()


def test_chain_restatement_is_the_reference_chain():
    # Four patches on 2 x 2 windows chained by the reference's SourceChain (nested seams, each
    # link's lattice over the patch before it).
    from terraingen_b200 import GridSpec

    z = dict(np.load(GOLDEN / "chain.npz"))
    g = grid_of(z["grid"])
    assert isinstance(g, GridSpec)
    wins = [tuple(int(x) for x in w) for w in z["windows"]]
    patches = [z[f"patch{k}"] for k in range(4)]
    for name in ("feather", "height", "slope"):
        _, width, decay = z[f"{name}_options"]
        got = S.chain(patches, wins, g, name, float(width), float(decay))
        want = z[f"{name}_heights"]
        if name == "feather":
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        else:
            assert np.abs(got.astype(np.float64) - want).max() <= 1e-6, name
