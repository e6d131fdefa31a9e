"""The oracle against the reference's own known answers (CPU only).

The restatement (oracle/restate.cpp) must reproduce the reference's golden vectors
(tests/golden/noise/kernels_test.cpp:21-42 of the reference) bit for bit, and the reference
CPU path built from its sources (oracle/_ref/libtgref.so) where it is available.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import harness as H
from conftest import grid_of


@pytest.fixture(scope="module")
def rs():
    if not H.available("libtgrestate.so"):
        H.build("restate")
    return H.restate()


def f32(hexstr: str) -> float:
    return float(np.float32(float.fromhex(hexstr)))


def test_pcg_golden(rs):
    # kernels_test.cpp:21-25
    assert rs.rs_pcg(0) == 129708002
    assert rs.rs_pcg(1) == 2831084092
    assert rs.rs_pcg(0xDEADBEEF) == 1730779506


def test_pcg3d_golden(rs):
    # kernels_test.cpp:27-29
    out = np.zeros(3, np.uint32)
    rs.rs_pcg3d(1, 2, 3, out.ctypes.data)
    assert list(out) == [4204755366, 1223881804, 1500469937]


@pytest.mark.parametrize("x,y,expected", [
    ("0x1p-2", "0x1.8p-1", "0x1.93a3e6p-4"),
    ("-0x1.9p+3", "0x1.9p+1", "-0x1.459948p-1"),
    ("0x1.f42666p+9", "-0x1.f56666p+7", "0x1.0de226p-1"),
])
def test_perlin2_golden(rs, x, y, expected):
    # kernels_test.cpp:31-35
    assert rs.rs_perlin2_f32(f32(x), f32(y), 1234) == f32(expected)


@pytest.mark.parametrize("x,y,expected", [
    ("0x0p+0", "0x0p+0", "0x1.822c5cp+3"),
    ("0x1.004p+9", "-0x1.001p+10", "-0x1.a18ed6p+0"),
    ("-0x1.77p+11", "0x1.000cp+12", "0x1.972ec2p+3"),
])
def test_fbm_golden(rs, x, y, expected):
    # kernels_test.cpp:37-42: FractalParams defaults (1000 m, 100 m, 8 octaves, 2, 0.5), seed 42
    got = rs.rs_fbm2_f32(f32(x), f32(y), 42, 1000.0, 100.0, 8, 2.0, 0.5)
    assert got == f32(expected)


def test_fbm_f64_close_to_f32(rs):
    # The FP64 form shares the lattice; it differs from the float form only by rounding.
    rng = np.random.default_rng(0)
    for x, y in rng.uniform(-3000, 3000, (200, 2)):
        a = rs.rs_fbm2_f32(float(np.float32(x)), float(np.float32(y)), 7, 512.0, 5.0, 8, 2.0, 0.5)
        b = rs.rs_fbm2_f64(float(np.float32(x)), float(np.float32(y)), 7, 512.0, 5.0, 8, 2.0, 0.5)
        assert abs(a - b) < 1e-5


def test_restated_grid_matches_fixture(rs, noise_fixture):
    # The fBm and DEM fixtures come from the reference CPU path (tests/golden/make_fixtures.py).
    for name in ("fbm", "dem", "far"):
        grid = grid_of(noise_fixture[f"{name}_grid"])
        fr = noise_fixture[f"{name}_fractals"].view(H.np.uint8)
        from terraingen_b200.layouts import FRACTAL
        f = fr.view(FRACTAL)[0]
        out = np.zeros((grid.height, grid.width), np.float32)
        rs.rs_fbm_grid_f32(grid.width, grid.height, grid.x0, grid.y0, grid.pixel, int(f["seed"]),
                           float(f["wavelength"]), float(f["amplitude"]), int(f["octaves"]),
                           float(f["lacunarity"]), float(f["gain"]),
                           float(noise_fixture[f"{name}_elevation"]), out.ctypes.data)
        expected = noise_fixture[f"{name}_heights"]
        assert np.array_equal(out.view(np.uint32), expected.view(np.uint32)), name


def test_crater_profile_f64_matches_reference_shape(rs):
    # Fassett-Thomson over the diameter: -0.181 D on the floor (x <= 0.2) unless the current depth
    # below the fresh rim is shallower, max(h, freshRim - currentDepth) (craters.h:338-362), and 0
    # beyond 1.5 radii.
    d = 10.0
    assert rs.rs_crater_profile_f64(0, 0, 0.5, d, 0.2, 0.04, 0.2, 0.04) == pytest.approx(-0.16 * d)
    assert rs.rs_crater_profile_f64(0, 0, 0.5, d, 0.2, 0.0, 0.2, 0.0) == pytest.approx(-0.181 * d)
    assert rs.rs_crater_profile_f64(0, 0, 7.6, d, 0.2, 0.04, 0.2, 0.04) == 0.0


@pytest.mark.skipif(not H.available("libtgref.so"), reason="reference build not present")
def test_reference_config1_checksum():
    # The 257^2 crater terrain through the reference CPU path: same bits on 1 and all threads
    # (the reference's determinism contract, apply_test.cpp:393), and the crater fixture's heights.
    from terraingen_b200 import centered

    ref = H.reference()
    scene = H.make_scene(centered(257, 257, 1.0), craters=H.config1_craters())
    one, _ = H.evaluate(ref, scene, 0, 1)
    many, _ = H.evaluate(ref, scene, 0, 0)
    assert np.array_equal(one.view(np.uint32), many.view(np.uint32))
    fixture = np.load(H.HERE.parent / "tests" / "golden" / "craters.npz")
    assert np.array_equal(one.view(np.uint32), fixture["config1_expected"].view(np.uint32))


def test_population_fixture_is_consistent():
    pop = np.load(H.HERE.parent / "tests" / "golden" / "population.npz")
    assert len(pop["id"]) > 1500
    assert np.all(pop["diameter"] >= 2.0) and np.all(pop["diameter"] <= 60.0)
    assert len(np.unique(pop["id"])) == len(pop["id"])
