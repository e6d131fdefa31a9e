"""The drop-in device inside the reference's own pipeline: Terrain::Evaluate with Backend::Cuda,
whose CudaCompute is the product's adapter (terraingen_b200/adapter/cuda_compute.cpp) on
libtgb200, against Backend::Cpu of the same build and the committed fixture."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(device):
    if not H.available("libtgref_cuda.so"):
        pytest.skip("oracle/_ref/libtgref_cuda.so was not built with the reference")
    return H.dropin()


def test_config1_through_reference_pipeline(dropin, crater_fixture):
    from terraingen_b200 import centered

    scene = H.make_scene(centered(257, 257, 1.0), craters=H.config1_craters())
    cpu, _ = H.evaluate(dropin, scene, 0, 1)
    gpu, _ = H.evaluate(dropin, scene, 1, 1)
    assert np.array_equal(cpu.view(np.uint32), crater_fixture["config1_expected"].view(np.uint32))
    err = np.abs(gpu.astype(np.float64) - cpu)
    assert err.max() <= 1e-3, err.max()


def test_noise_layer_through_reference_pipeline(dropin, noise_fixture):
    from terraingen_b200 import centered
    from terraingen_b200.layouts import fractal

    g = centered(70, 50, 1.0, 10.0, 20.0)
    src = np.array([fractal(seed=21, wavelength=400.0, amplitude=30.0, octaves=6)])
    lay = np.array([fractal(seed=22, wavelength=60.0, amplitude=2.0, octaves=4),
                    fractal(seed=23, wavelength=25.0, amplitude=0.5, octaves=3, basis=1)])
    scene = H.make_scene(g, source_fractals=src, layer_fractals=lay)
    gpu, _ = H.evaluate(dropin, scene, 1, 1)
    assert np.array_equal(gpu.view(np.uint32), noise_fixture["layer_expected"].view(np.uint32))


def test_craters_on_a_body_through_reference_pipeline(dropin):
    # A site on a sphere of the Moon's radius: the reference dispatches its crater kernel with
    # frames and split points (ShapeCratersOnBody); the adapter runs tg_craters_apply_body.
    import importlib.util

    from conftest import GOLDEN

    spec = importlib.util.spec_from_file_location("body_cases", GOLDEN / "body_cases.py")
    cases = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cases)
    want = np.load(GOLDEN / "body.npz")["expected"]
    scene = cases.scene()
    cpu, _ = H.evaluate(dropin, scene, 0, 1)
    gpu, _ = H.evaluate(dropin, scene, 1, 1)
    assert np.array_equal(cpu.view(np.uint32), want.view(np.uint32))
    assert np.count_nonzero(want) > 5000
    err = np.abs(gpu.astype(np.float64) - cpu)
    assert err.max() <= 1e-3, err.max()


def test_crater_datums_on_a_body_through_reference_pipeline(dropin):
    # Plane datums on a sphere: the reference fits them with its body datum kernel
    # (crater_body_datums.slang), which the adapter runs as tg_crater_body_datums.
    import importlib.util

    from conftest import GOLDEN

    spec = importlib.util.spec_from_file_location("body_cases", GOLDEN / "body_cases.py")
    cases = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cases)
    want = np.load(GOLDEN / "body.npz")["datum_expected"]
    scene = cases.scene(datum=1)
    cpu, _ = H.evaluate(dropin, scene, 0, 1)
    gpu, _ = H.evaluate(dropin, scene, 1, 1)
    assert np.array_equal(cpu.view(np.uint32), want.view(np.uint32))
    err = np.abs(gpu.astype(np.float64) - cpu)
    assert err.max() <= 1e-3, err.max()


def test_terrain_through_hooked_reference_pipeline(dropin):
    # The synthetic terrain's stack (fBm source, Config-2 craters with peaks and terraces,
    # boulder domes) through the reference's Terrain::Evaluate on Backend::Cuda: the drop-in build
    # runs its source fill (tg_noise_source), crater shaping (the adapter) and boulder bake
    # (tg_boulders_bake) on the device, and the population and records stay on the reference's
    # CPU path. The result is the CPU backend's within 1e-3 m.
    from terraingen_b200.workloads import terrain4097_reference_scene

    grid, fr, craters, boulders = terrain4097_reference_scene(257)
    scene = H.make_scene(grid, source_fractals=fr, craters=craters, boulders=boulders)
    before = H.hook_calls(dropin)
    gpu, _ = H.evaluate(dropin, scene, 1, 1)
    assert H.hook_calls(dropin) - before >= 2  # the source and the boulders ran on the device
    cpu, _ = H.evaluate(dropin, scene, 0, 1)
    err = np.abs(gpu.astype(np.float64) - cpu)
    assert err.max() <= 1e-3, err.max()
    assert np.count_nonzero(gpu != gpu[0, 0]) > 0.9 * gpu.size


@pytest.mark.parametrize("name", ["dem5m", "exact", "tenfold", "tenfold_cr"])
def test_ds_through_hooked_reference_pipeline(dropin, name):
    # The reference's DiamondSquareUpsampler behind a RasterSource on Backend::Cuda: the drop-in
    # build's hook hands the refinement to tg_ds_refine, which gives the committed fixture (the
    # reference's CPU refinement) within 1e-3 m.
    from conftest import GOLDEN, grid_of

    fx = dict(np.load(GOLDEN / "ds.npz"))
    pg = grid_of(fx[f"{name}_post_grid"])
    grid = grid_of(fx[f"{name}_grid"])
    fd, scale, seed, interp = fx[f"{name}_options"]
    before = H.hook_calls(dropin)
    gpu, _ = H.diamond_square(dropin, fx[f"{name}_posts"], pg, grid, fd, scale, int(seed),
                              int(interp), 1, backend=1)
    assert H.hook_calls(dropin) - before >= 1
    err = np.abs(gpu.astype(np.float64) - fx[f"{name}_expected"])
    assert err.max() <= 1e-3, (name, err.max())
