"""tg_noise_source_body (SyntheticSource on a sphere: FractalStackAt on a body, Fractal3 with
double-split lattice points) against the reference CPU path's heights (tests/golden/body_noise.npz,
tests/golden/body_noise_cases.py): every basis and fractal type, blends and a warp, at two sites,
bit for bit, from host arrays and device tensors."""

from __future__ import annotations

import importlib.util

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location("body_noise_cases", GOLDEN / "body_noise_cases.py")
CASES = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(CASES)
ALL = CASES.cases()
WANT = np.load(GOLDEN / "body_noise.npz")


@pytest.mark.parametrize("site", sorted(ALL["sites"]))
@pytest.mark.parametrize("stack", sorted(ALL["stacks"]))
def test_body_source_is_the_reference(device, stack, site):
    grid = ALL["sites"][site]
    fr = np.array(ALL["stacks"][stack])
    host = np.zeros((grid.height, grid.width), np.float32)
    device.noise_source_body(fr, grid, CASES.RADIUS, host, elevation=1000.0)
    want = WANT[f"{stack}_{site}"]
    assert np.array_equal(host.view(np.uint32), want.view(np.uint32)), \
        float(np.abs(host.astype(np.float64) - want).max())


def test_body_source_from_device_tensors(device):
    import torch

    grid = ALL["sites"]["equator"]
    fr = np.array(ALL["stacks"]["warped"])
    out = torch.empty((grid.height, grid.width), dtype=torch.float32, device="cuda")
    device.noise_source_body(fr, grid, CASES.RADIUS, out, elevation=1000.0)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32),
                          WANT["warped_equator"].view(np.uint32))


def test_body_source_refuses_a_bad_radius(device):
    from terraingen_b200 import TgError

    grid = ALL["sites"]["equator"]
    with pytest.raises(TgError):
        device.noise_source_body(np.array(ALL["stacks"]["perlin_fbm"]), grid, 0.0,
                                 np.zeros((grid.height, grid.width), np.float32))
