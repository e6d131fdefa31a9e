"""GPU tests of the seam solve (tg_seam_solve, tg_seam_fill) against the reference's seams
(tests/golden/seams.npz) and the seam restatement (oracle/seams.py).

- Feather: the field bit for bit (the chamfer distances' float recurrences in the reference's
  order).
- Height / Slope: within 1e-4 m of the reference's field (both solve the same system to a
  residual of 1e-10; the device runs FP64 conjugate gradients with an FP32 multigrid).
- Filling a grid's gaps from the reference's field: the chain's heights bit for bit, on the
  rasters' grid and on a finer one; from the device's own field within 1e-4 m.
- Host and device memory give the same bits; no field where the earlier source has data at
  every post or at none, or with mode none.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, grid_of
from oracle import seams as S

pytestmark = pytest.mark.gpu

CASES = [(scene, mode) for scene in ("hole", "patch") for mode in ("feather", "height", "slope")]


@pytest.fixture(scope="module")
def z():
    return dict(np.load(GOLDEN / "seams.npz"))


def _solve(device, z, key, mode, **kw):
    lat = z[f"{key}_lattice"]
    _, width, decay = z[f"{key}_options"]
    return device.seam_solve(z[f"{key}_data"], z[f"{key}_difference"], float(lat[3]),
                             float(-lat[7]), mode, width=float(width),
                             decay_length=float(decay), **kw)


def _lattice_grid(z, key):
    from terraingen_b200.device import GridSpec

    lat = z[f"{key}_lattice"]
    return GridSpec(int(lat[0]), int(lat[1]), float(lat[2]), float(lat[5]), float(lat[3]))


@pytest.mark.parametrize("scene", ["hole", "patch"])
def test_feather_field_is_bit_exact(device, z, scene):
    key = f"{scene}_feather"
    field, _ = _solve(device, z, key, "feather")
    want = z[f"{key}_field"]
    assert np.array_equal(field.view(np.uint32), want.view(np.uint32)), np.abs(field - want).max()


@pytest.mark.parametrize("scene,mode", [(s, m) for s in ("hole", "patch")
                                        for m in ("height", "slope")])
def test_screened_field_within_tolerance(device, z, scene, mode):
    key = f"{scene}_{mode}"
    field, stats = _solve(device, z, key, mode)
    want = z[f"{key}_field"]
    lat = z[f"{key}_lattice"]
    d, _ = S.distances(z[f"{key}_data"], float(lat[3]), float(-lat[7]))
    unknowns = S.unknowns(z[f"{key}_data"], d, 3.0 * float(z[f"{key}_options"][2]))
    assert stats["unknowns"] == int(unknowns.sum())
    assert stats["iterations"] < 200, stats
    err = np.abs(field.astype(np.float64) - want).max()
    assert err <= 1e-4, (err, stats)
    assert np.array_equal(field[~unknowns].view(np.uint32), want[~unknowns].view(np.uint32))


@pytest.mark.parametrize("scene,mode", CASES)
def test_fill_from_reference_field_is_the_chain(device, z, scene, mode):
    key = f"{scene}_{mode}"
    lattice = _lattice_grid(z, key)
    for prefix, grid in (("", z[f"{scene}_grid"]), ("fine_", z[f"{scene}_fine_grid"])):
        heights = z[f"{scene}_{prefix}earlier"].copy()
        device.seam_fill(z[f"{key}_field"], lattice, z[f"{scene}_{prefix}later"], grid_of(grid),
                         heights)
        want = z[f"{key}_{prefix}chain"]
        assert np.array_equal(heights.view(np.uint32), want.view(np.uint32)), prefix


@pytest.mark.parametrize("scene,mode", CASES)
def test_solve_then_fill_within_tolerance(device, z, scene, mode):
    key = f"{scene}_{mode}"
    field, _ = _solve(device, z, key, mode)
    lattice = _lattice_grid(z, key)
    heights = z[f"{scene}_fine_earlier"].copy()
    device.seam_fill(field, lattice, z[f"{scene}_fine_later"], grid_of(z[f"{scene}_fine_grid"]),
                     heights)
    want = z[f"{key}_fine_chain"]
    err = np.abs(heights.astype(np.float64) - want).max()
    assert err <= 1e-4, err


def test_device_memory_matches_host(device, z):
    import torch

    key = "hole_slope"
    host, _ = _solve(device, z, key, "slope")
    data = torch.from_numpy(z[f"{key}_data"]).cuda()
    diff = torch.from_numpy(z[f"{key}_difference"]).cuda()
    lat = z[f"{key}_lattice"]
    field, _ = device.seam_solve(data, diff, float(lat[3]), float(-lat[7]), "slope",
                                 decay_length=float(z[f"{key}_options"][2]))
    torch.cuda.synchronize()
    assert np.array_equal(field.cpu().numpy().view(np.uint32), host.view(np.uint32))
    # The same solve twice: the same bits (deterministic reductions).
    again, _ = _solve(device, z, key, "slope")
    assert np.array_equal(again.view(np.uint32), host.view(np.uint32))
    # Fill on the device.
    heights = torch.from_numpy(z["hole_fine_earlier"].copy()).cuda()
    later = torch.from_numpy(z["hole_fine_later"]).cuda()
    device.seam_fill(field, _lattice_grid(z, key), later, grid_of(z["hole_fine_grid"]), heights)
    torch.cuda.synchronize()
    want = z["hole_fine_earlier"].copy()
    device.seam_fill(host, _lattice_grid(z, key), z["hole_fine_later"],
                     grid_of(z["hole_fine_grid"]), want)
    assert np.array_equal(heights.cpu().numpy().view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("mode", ["feather", "height", "slope"])
def test_no_field_without_a_gap_or_without_data(device, mode):
    rng = np.random.default_rng(1)
    diff = rng.standard_normal((40, 50)).astype(np.float32)
    for data in (np.ones((40, 50), np.uint8), np.zeros((40, 50), np.uint8)):
        field, st = device.seam_solve(data, diff, 1.0, 1.0, mode, width=5.0, decay_length=3.0)
        assert not field.any() and st["unknowns"] == 0
    data = np.ones((40, 50), np.uint8)
    data[10:20, 10:30] = 0
    field, _ = device.seam_solve(data, diff, 1.0, 1.0, "none")
    assert not field.any()


@pytest.mark.parametrize("mode", ["feather", "height", "slope"])
def test_small_and_ragged_lattices(device, mode):
    # Lattices narrower than the border and band, non-square posts, gaps at the edges: against
    # the restatement.
    rng = np.random.default_rng(7)
    for h, w, dx, dy in ((5, 6, 1.0, 1.0), (9, 40, 0.5, 2.0), (33, 17, 3.0, 1.5), (70, 90, 1.0, 1.0)):
        data = (rng.random((h, w)) > 0.35).astype(np.uint8)
        data[:, : w // 3] = 0
        diff = np.where(data != 0, rng.standard_normal((h, w)), np.nan).astype(np.float32)
        diff[data != 0] += 3.0
        field, _ = device.seam_solve(data, diff, dx, dy, mode, width=4.0, decay_length=2.5)
        if mode == "feather":
            want = S.feather(data, diff, dx, dy, 4.0)
            assert np.array_equal(field.view(np.uint32), want.view(np.uint32)), (h, w)
        else:
            want = S.solve(data, diff, dx, dy, mode, 2.5)
            err = np.abs(field.astype(np.float64) - want).max()
            assert err <= 1e-4, (h, w, err)


def test_refuses_bad_options(device):
    from terraingen_b200 import TgError

    data = np.ones((8, 8), np.uint8)
    diff = np.zeros((8, 8), np.float32)
    with pytest.raises(TgError):
        device.seam_solve(data, diff, 0.0, 1.0, "height")
    with pytest.raises(TgError):
        device.seam_solve(data, diff, 1.0, 1.0, "feather", width=-1.0)
    with pytest.raises(TgError):
        device.seam_solve(data, diff, 1.0, 1.0, "slope", levels=0)


@pytest.mark.parametrize("scene,mode", CASES)
def test_samples_are_the_reference_lattice(device, z, scene, mode):
    # The lattice pads the rasters' grid by ceil(reach / spacing) + 3 posts on every side.
    import math

    key = f"{scene}_{mode}"
    g = grid_of(z[f"{scene}_grid"])
    lat = z[f"{key}_lattice"]
    pad = (int(lat[0]) - g.width) // 2
    _, width, decay = z[f"{key}_options"]
    assert pad == math.ceil((width if mode == "feather" else 3.0 * decay) / g.pixel) + 3
    data, diff = device.seam_samples(z[f"{scene}_earlier"], z[f"{scene}_later"], g, -pad, -pad,
                                     int(lat[0]), int(lat[1]))
    assert np.array_equal(data, z[f"{key}_data"])
    assert np.array_equal(diff.view(np.uint32), z[f"{key}_difference"].view(np.uint32))


@pytest.mark.parametrize("mode", ["feather", "height"])
def test_wide_reach(device, mode):
    # A reach wider than the lattice: every tile's window is the whole lattice.
    rng = np.random.default_rng(12)
    h, w = 240, 260
    data = np.ones((h, w), np.uint8)
    yy, xx = np.mgrid[0:h, 0:w]
    data[((yy - 120) / 70.0) ** 2 + ((xx - 140) / 90.0) ** 2 < 1.0] = 0
    diff = np.where(data != 0, 2.0 + 0.01 * xx - 0.02 * yy + 0.1 * rng.standard_normal((h, w)),
                    np.nan).astype(np.float32)
    field, _ = device.seam_solve(data, diff, 0.5, 0.5, mode, width=120.0, decay_length=40.0)
    if mode == "feather":
        want = S.feather(data, diff, 0.5, 0.5, 120.0)
        assert np.array_equal(field.view(np.uint32), want.view(np.uint32))
    else:
        want = S.solve(data, diff, 0.5, 0.5, mode, 40.0)
        assert np.abs(field.astype(np.float64) - want).max() <= 1e-4


@pytest.mark.parametrize("mode", ["feather", "height"])
def test_windows_wider_than_shared_memory(device, mode):
    # A window of 13,000 columns: the rows the distance warps hand down are kept in device memory
    # instead of shared memory.
    rng = np.random.default_rng(21)
    h, w = 40, 13000
    data = np.ones((h, w), np.uint8)
    data[10:30, 6400:6600] = 0
    xx = np.arange(w)[None, :]
    diff = np.where(data != 0, 1.0 + 1e-4 * xx + 0.1 * rng.standard_normal((h, w)),
                    np.nan).astype(np.float32)
    field, st = device.seam_solve(data, diff, 1.0, 1.0, mode, width=7000.0, decay_length=2200.0)
    if mode == "feather":
        want = S.feather(data, diff, 1.0, 1.0, 7000.0)
        assert np.array_equal(field.view(np.uint32), want.view(np.uint32))
    else:
        assert st["unknowns"] == 20 * 200
        want = S.solve(data, diff, 1.0, 1.0, mode, 2200.0)
        assert np.abs(field.astype(np.float64) - want).max() <= 1e-4


@pytest.mark.parametrize("mode", ["feather", "height", "slope"])
def test_patch_chain_is_the_reference_chain(device, mode):
    # PatchChain (samples, solve and fill per link, on the device) against the reference's
    # SourceChain of the same four patches.
    import torch

    from terraingen_b200.chain import PatchChain, Seams, Window

    z = dict(np.load(GOLDEN / "chain.npz"))
    g = grid_of(z["grid"])
    wins = [Window(*(int(x) for x in w)) for w in z["windows"]]
    _, width, decay = z[f"{mode}_options"]
    chain = PatchChain(device, g, wins, Seams(mode, width=float(width),
                                              decay_length=float(decay)))
    patches = [torch.from_numpy(z[f"patch{k}"]).cuda() for k in range(4)]
    got = chain.compose(patches).cpu().numpy()
    want = z[f"{mode}_heights"]
    assert len(chain.solves) == 3
    if mode == "feather":
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        assert np.abs(got.astype(np.float64) - want).max() <= 1e-4


def test_fill_window_is_the_fill_within_it(device, z):
    # A window of the grid: the same cells as the whole fill inside it, nothing outside.
    key = "hole_height"
    lattice = _lattice_grid(z, key)
    g = grid_of(z["hole_fine_grid"])
    whole = z["hole_fine_earlier"].copy()
    device.seam_fill(z[f"{key}_field"], lattice, z["hole_fine_later"], g, whole)
    part = z["hole_fine_earlier"].copy()
    c0, r0, w, h = 17, 9, 101, 77
    device.seam_fill(z[f"{key}_field"], lattice, z["hole_fine_later"], g, part,
                     window=(c0, r0, w, h))
    inside = np.zeros(part.shape, bool)
    inside[r0:r0 + h, c0:c0 + w] = True
    assert np.array_equal(part[inside].view(np.uint32), whole[inside].view(np.uint32))
    before = z["hole_fine_earlier"]
    assert np.array_equal(part[~inside].view(np.uint32), before[~inside].view(np.uint32))
    assert np.count_nonzero(part[inside] != before[inside]) > 100
