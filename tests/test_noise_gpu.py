"""GPU parity of the noise kernels against the reference CPU path (bit-exact) and the restated
oracle, through the C ABI."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import grid_of
from terraingen_b200.layouts import FRACTAL, NOISE_LAYER_KERNEL

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["fbm", "dem", "stack", "far"])
def test_noise_source_bit_exact(device, noise_fixture, name):
    grid = grid_of(noise_fixture[f"{name}_grid"])
    fractals = noise_fixture[f"{name}_fractals"].view(FRACTAL)
    heights = np.zeros((grid.height, grid.width), np.float32)
    device.noise_source(fractals, grid, heights, float(noise_fixture[f"{name}_elevation"]))
    expected = noise_fixture[f"{name}_heights"]
    diff = np.abs(heights.astype(np.float64) - expected)
    assert np.array_equal(heights.view(np.uint32), expected.view(np.uint32)), (
        f"{name}: {np.count_nonzero(diff)} cells differ, max {diff.max()}")


def test_noise_layer_rows_bit_exact(device, noise_fixture):
    # The strip the reference's NoiseLayer hands RunKernel (captured through the drop-in device).
    kernel = noise_fixture["layer_kernel"].view(NOISE_LAYER_KERNEL)[0]
    xs = noise_fixture["layer_xs"].view(np.float32)
    ys = noise_fixture["layer_ys"].view(np.float32)
    heights = noise_fixture["layer_heights"].view(np.float32).copy()
    device.noise_layer_rows(kernel, xs, ys, heights)
    expected = noise_fixture["layer_expected"].reshape(-1)
    assert np.array_equal(heights.view(np.uint32), expected.view(np.uint32))


def test_noise_layer_grid_matches_rows(device, noise_fixture):
    # The grid form computes the same positions on the device from the transform.
    from terraingen_b200 import centered

    kernel = noise_fixture["layer_kernel"].view(NOISE_LAYER_KERNEL)[0]
    grid = centered(70, 50, 1.0, 10.0, 20.0)
    base = noise_fixture["layer_heights"].view(np.float32).reshape(grid.height, grid.width)
    heights = base.copy()
    device.noise_layer(kernel, grid, heights, origin=(0.0, 0.0))
    expected = noise_fixture["layer_expected"]
    assert np.array_equal(heights.view(np.uint32), expected.view(np.uint32))


def test_noise_layer_skips_nodata(device):
    from terraingen_b200 import centered
    from terraingen_b200.layouts import fractal, noise_layer_kernel

    grid = centered(33, 17, 1.0)
    kernel = noise_layer_kernel([fractal(seed=3, wavelength=50.0, amplitude=2.0)])
    heights = np.zeros((grid.height, grid.width), np.float32)
    heights[3, 5] = np.nan
    heights[7, 9] = -9999.0
    a = heights.copy()
    device.noise_layer(kernel, grid, a, nodata=(1, 0.0))
    assert np.isnan(a[3, 5]) and a[7, 9] != -9999.0
    b = heights.copy()
    device.noise_layer(kernel, grid, b, nodata=(2, -9999.0))
    assert b[7, 9] == -9999.0


def test_probe_against_restatement(device):
    from oracle import harness as H

    rs = H.restate()
    rng = np.random.default_rng(1)
    xy = np.concatenate([rng.uniform(-2000, 2000, (256, 2)),
                         rng.uniform(-5, 5, (64, 2))]).astype(np.float32)
    hashes, values = device.noise_probe(xy, 1234)
    for i, (x, y) in enumerate(xy):
        assert hashes[i, 0] == rs.rs_pcg(i)
        h3 = np.zeros(3, np.uint32)
        rs.rs_pcg3d(int(x.view(np.uint32)), int(y.view(np.uint32)), 1234, h3.ctypes.data)
        assert list(hashes[i, 1:]) == list(h3)
        assert values[i, 0] == np.float32(rs.rs_perlin2_f32(float(x), float(y), 1234))
        fbm = rs.rs_fbm2_f32(float(x), float(y), 1234, 1000.0, 100.0, 8, 2.0, 0.5)
        assert values[i, 6] == np.float32(fbm)


def test_probe_golden_vectors(device):
    # The reference's golden vectors (tests/golden/noise/kernels_test.cpp:31-42) on the GPU.
    def f(h):
        return np.float32(float.fromhex(h))

    xy = np.array([[f("0x1p-2"), f("0x1.8p-1")], [f("-0x1.9p+3"), f("0x1.9p+1")],
                   [f("0x1.f42666p+9"), f("-0x1.f56666p+7")]], np.float32)
    _, values = device.noise_probe(xy, 1234)
    assert list(values[:, 0]) == [f("0x1.93a3e6p-4"), f("-0x1.459948p-1"), f("0x1.0de226p-1")]
    # Simplex and value noise goldens (kernels_test.cpp:44-52).
    assert values[0, 1] == f("0x1.bac986p-4") and values[1, 1] == f("0x1.88e9b6p-2")
    assert values[0, 2] == f("-0x1.0ed85ap-1") and values[1, 2] == f("-0x1.a6cecp-2")
    assert values[0, 3] == f("0x1.0f7b3p-1") and values[0, 4] == f("0x1.2e7808p-1")
    xy = np.array([[0.0, 0.0], [f("0x1.004p+9"), f("-0x1.001p+10")],
                   [f("-0x1.77p+11"), f("0x1.000cp+12")]], np.float32)
    _, values = device.noise_probe(xy, 42)
    assert list(values[:, 6]) == [f("0x1.822c5cp+3"), f("-0x1.a18ed6p+0"), f("0x1.972ec2p+3")]
    # Ridged, billow, hybrid at the second point (kernels_test.cpp:54-65).
    assert values[1, 7] == f("0x1.8fd9ap+5")
    assert values[1, 8] == f("-0x1.26132cp+6")
    assert values[1, 9] == f("0x1.58502ap+5")


def test_noise_device_memory_matches_host(device):
    import torch

    from terraingen_b200 import centered
    from terraingen_b200.layouts import fractal

    grid = centered(300, 200, 0.5, 50.0, 50.0)
    fr = np.array([fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)])
    host = np.zeros((grid.height, grid.width), np.float32)
    device.noise_source(fr, grid, host)
    dev = torch.zeros((grid.height, grid.width), dtype=torch.float32, device="cuda")
    device.noise_source(fr, grid, dev)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))
