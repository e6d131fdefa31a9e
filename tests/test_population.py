"""Crater populations and kernel batches built by the product's host code, bit-exact against the
reference (CPU only): the population fixture and the batches the reference hands its GPU
backend (tests/golden/make_fixtures.py)."""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import harness as H
from terraingen_b200 import _native as N, centered
from terraingen_b200.layouts import CRATER_RECORD, CRATER_SHAPE_KERNEL


def population(fields: dict, margin_radii=0.0, min_resolved=0.0) -> N.Population:
    return N.Population(seed=fields["seed"], sfd_coefficient=fields["sfdCoefficient"],
                        sfd_exponent=fields.get("sfdExponent", 2.0),
                        min_diameter=fields["minDiameter"], max_diameter=fields["maxDiameter"],
                        lifetime_gyr=fields.get("lifetimeGyr", 1.0),
                        depth_ratio=fields.get("depthRatio", 0.2),
                        rim_ratio=fields.get("rimRatio", 0.04), cutoff_depth_ratio=0.04,
                        cell_size_factor=16.0, margin_radii=margin_radii,
                        min_resolved_diameter=min_resolved)


def generate(pop: N.Population, region) -> dict:
    lib = N.library()
    region = np.asarray(region, np.float64)
    n = C.c_size_t()
    N.check(lib.tg_crater_generate(C.byref(pop), region.ctypes.data, None, None, None, None, None,
                                   0, C.byref(n)))
    out = {k: np.zeros(n.value) for k in ("x", "y", "diameter", "age")}
    out["id"] = np.zeros(n.value, np.uint64)
    N.check(lib.tg_crater_generate(C.byref(pop), region.ctypes.data, out["x"].ctypes.data,
                                   out["y"].ctypes.data, out["diameter"].ctypes.data,
                                   out["age"].ctypes.data, out["id"].ctypes.data, n.value,
                                   C.byref(n)))
    return out


def batch(pop: N.Population, profile: int, irregular: int, grid, **shaping):
    lib = N.library()
    shp = N.Shaping(profile=profile, irregular=irregular, **shaping)
    g = grid.native()
    nr, nd = C.c_size_t(), C.c_size_t()
    N.check(lib.tg_crater_batch(C.byref(pop), C.byref(shp), C.byref(g), None, None, 0, None, 0,
                                None, C.byref(nr), C.byref(nd)))
    k = np.zeros((), CRATER_SHAPE_KERNEL)
    rec = np.zeros(nr.value, CRATER_RECORD)
    data = np.zeros(nd.value, np.float32)
    foot = np.zeros(3 * nr.value)
    N.check(lib.tg_crater_batch(C.byref(pop), C.byref(shp), C.byref(g), k.ctypes.data,
                                rec.ctypes.data, nr.value, data.ctypes.data, nd.value,
                                foot.ctypes.data, C.byref(nr), C.byref(nd)))
    return k, rec, data, foot


def test_population_matches_reference_fixture():
    # The 257^2 scene's layer over its grid: CraterLayer::Craters with the layer's margin
    # (reach 1.5 x the default irregular outline's largest stretch) and 2-sample resolution.
    want = np.load(GOLDEN / "population.npz")
    margin = 1.5 * (1 + 0.03 * math.sqrt(22)) * math.sqrt(1.5)
    got = generate(population(H.config1_craters(), margin, 2.0), (-128.5, -128.5, 128.5, 128.5))
    for key in ("x", "y", "diameter", "age", "id"):
        assert np.array_equal(got[key], want[key]), key


def test_batch_matches_captured_config1(crater_fixture):
    k, rec, data, _ = batch(population(H.config1_craters()), 0, 1, centered(257, 257, 1.0))
    assert k.tobytes() == crater_fixture["config1_kernel"].tobytes()
    assert rec.tobytes() == crater_fixture["config1_records"].tobytes()
    assert data.tobytes() == crater_fixture["config1_data"].tobytes()


def test_batch_matches_captured_mpd(crater_fixture):
    # Martin-Parkes-Dunstan with plain (round) outlines on an off-center 0.5 m grid.
    # The "mpd" scene of tests/golden/make_fixtures.py.
    grid = centered(160, 144, 0.5, 40.0, -25.0)
    fields = dict(seed=5, sfdCoefficient=4e-2, minDiameter=1.0, maxDiameter=40.0)
    k, rec, data, _ = batch(population(fields), 1, 0, grid)
    assert k.tobytes() == crater_fixture["mpd_kernel"].tobytes()
    assert rec.tobytes() == crater_fixture["mpd_records"].tobytes()
    assert data.tobytes() == crater_fixture["mpd_data"].tobytes()


def test_batch_matches_captured_complex(crater_fixture):
    # Complex craters over Fassett-Thomson (lowered transition) with the default apply: massif
    # peaks on every complex crater and wall terraces from 80 m, records and data bit-exact with
    # what the reference hands its GPU backend (AppendKernelTerraces, AppendKernelPeaks). The
    # scene's rim smoothing is a kernel option only; every other kernel field matches.
    grid = centered(192, 192, 2.0)
    fields = dict(seed=9, sfdCoefficient=0.6, minDiameter=8.0, maxDiameter=300.0)
    k, rec, data, _ = batch(population(fields), 2, 1, grid, transition_diameter=60.0,
                            terrace_onset=80.0, terrace_full=200.0, terrace_min_freshness=0.3)
    want = crater_fixture["complex_records"].view(CRATER_RECORD)
    assert np.any(rec["peakCount"] > 0) and np.any(rec["terraceCount"] > 0)
    assert rec.tobytes() == want.tobytes()
    assert data.tobytes() == crater_fixture["complex_data"].tobytes()
    wk = crater_fixture["complex_kernel"].view(CRATER_SHAPE_KERNEL).reshape(())
    for name in CRATER_SHAPE_KERNEL.names:
        if name != "rimSigma":
            assert np.asarray(k[name]).tobytes() == np.asarray(wk[name]).tobytes(), name


def test_batch_rejects_bad_shaping():
    lib = N.library()
    pop = population(dict(seed=1, sfdCoefficient=0.1, minDiameter=2.0, maxDiameter=20.0))
    g = centered(32, 32, 1.0).native()
    nr, nd = C.c_size_t(), C.c_size_t()
    for shaping in (N.Shaping(profile=4), N.Shaping(profile=2, transition_diameter=0.0),
                    N.Shaping(profile=0, irregular=1, terrace_onset=100.0, terrace_full=50.0),
                    N.Shaping(profile=0, irregular=1, terrace_onset=100.0, terrace_full=200.0,
                              terrace_min_freshness=1.0)):
        assert lib.tg_crater_batch(C.byref(pop), C.byref(shaping), C.byref(g), None, None, 0,
                                   None, 0, None, C.byref(nr), C.byref(nd)) == 1


@pytest.mark.skipif(not H.available("libtgref_capture.so"), reason="reference build not present")
@pytest.mark.parametrize("cx,cy", [(300.0, -450.0), (-700.0, 820.0)])
def test_config2_window_matches_reference_live(cx, cy):
    # A window of the synthetic 4097^2 terrain's crater layer with its peaks and terraces mapped
    # onto the reference's options (terraingen_b200.workloads): the kernel, records and data the
    # reference's CraterLayer hands its GPU backend, captured live, against tg_crater_batch.
    from terraingen_b200 import workloads as W

    grid = centered(257, 257, 0.5, cx, cy)
    _, _, craters, _ = W.terrain4097_reference_scene(257)
    cap = H.capture()
    H.evaluate(cap, H.make_scene(grid, craters=craters), 1, 1)
    call = [c for c in H.captured(cap) if c["kind"] == 2][-1]
    area = (4097 * 0.5) ** 2
    coefficient = 200000.0 / (area * (1.0 ** -2.0 - 500.0 ** -2.0))
    k, rec, data, _ = W.crater_batch(W.crater_population(7, coefficient, 1.0, 500.0), grid,
                                     shaping=W.config2_shaping())
    assert np.any(rec["peakCount"] > 0)
    assert k.tobytes() == call["kernel"].tobytes()
    assert rec.tobytes() == call["records"].tobytes()
    assert data.tobytes() == call["data"].tobytes()


def test_population_deterministic_and_tiled():
    # Regions that tile a larger one draw the same craters (population_test.cpp:86-130): every
    # crater of the whole region centered in a tile appears in that tile's draw.
    fields = dict(seed=9, sfdCoefficient=0.05, minDiameter=1.0, maxDiameter=80.0)
    whole = generate(population(fields), (0.0, 0.0, 400.0, 400.0))
    again = generate(population(fields), (0.0, 0.0, 400.0, 400.0))
    assert np.array_equal(whole["id"], again["id"])
    ids = set()
    for x0 in (0.0, 200.0):
        for y0 in (0.0, 200.0):
            part = generate(population(fields), (x0, y0, x0 + 200.0, y0 + 200.0))
            ids |= set(part["id"].tolist())
    assert ids == set(whole["id"].tolist())


def test_population_rejects_bad_ranges():
    lib = N.library()
    pop = population(dict(seed=1, sfdCoefficient=0.1, minDiameter=5.0, maxDiameter=2.0))
    region = np.zeros(4)
    n = C.c_size_t()
    assert lib.tg_crater_generate(C.byref(pop), region.ctypes.data, None, None, None, None, None,
                                  0, C.byref(n)) == 1


@pytest.mark.skipif(not H.available("libtgref.so"), reason="reference build not present")
@pytest.mark.parametrize("seed,coefficient,lo,hi", [(2, 0.3, 1.0, 30.0), (77, 2.0, 0.5, 8.0)])
def test_population_matches_reference_live(seed, coefficient, lo, hi):
    # Denser draws (Poisson means above 10 take the PTRS branch) against the reference itself.
    fields = dict(seed=seed, sfdCoefficient=coefficient, minDiameter=lo, maxDiameter=hi,
                  profile=1, applyPreset=1)
    scene = H.make_scene(centered(100, 100, 0.5), craters=fields)
    region = (-30.0, -20.0, 45.0, 35.0)
    want = H.craters(H.reference(), scene, region, 0.0)
    got = generate(population(fields, margin_radii=2.0, min_resolved=0.0), region)
    for key in ("x", "y", "diameter", "age", "id"):
        assert np.array_equal(got[key], want[key]), key


# --- boulders (tg_boulder_generate) -------------------------------------------------------------

BOULDER_SCENES = {
    # (seed, coefficient, height ratio bounds, burial bounds), as tests/golden/make_fixtures.py
    # builds the reference's layers: exponent 2.5 on [0.2, 3] m.
    "dense": (1, 0.5, (0.5, 0.5), (0.0, 0.0)),
    "fine": (4, 0.3, (0.4, 0.4), (0.0, 0.0)),
    "posed": (9, 0.4, (0.3, 0.7), (0.1, 0.4)),
}


@pytest.mark.parametrize("name", sorted(BOULDER_SCENES))
def test_boulders_are_the_references(name):
    # The boulders the reference's BoulderLayer draws into the fixture grid (candidates from the
    # summed candidate SFD inverted numerically, thinning, pose and burial draws, resolution
    # weights): bit for bit, in its order.
    from terraingen_b200 import GridSpec
    from terraingen_b200.workloads import boulder_population, generate_boulders

    z = np.load(GOLDEN / "boulders.npz")
    g = z[f"{name}_grid"]
    grid = GridSpec(int(g[0]), int(g[1]), float(g[2]), float(g[3]), float(g[4]))
    seed, coefficient, ratio, burial = BOULDER_SCENES[name]
    got = generate_boulders(boulder_population(seed, coefficient, height_ratio=ratio,
                                               burial=burial), grid)
    want = z[f"{name}_boulders"]
    assert len(want) > 1000
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_boulder_generate_refuses_bad_input():
    from terraingen_b200.workloads import boulder_population

    lib = N.library()
    region = np.array([0.0, 0.0, 10.0, 10.0])
    n = C.c_size_t()
    pop = boulder_population(1, 0.5, dmin=3.0, dmax=0.2)
    assert lib.tg_boulder_generate(C.byref(pop), region.ctypes.data, 0.5, None, 0,
                                   C.byref(n)) == 1  # TG_ERROR_ARGUMENT
    pop = boulder_population(1, 0.5)
    assert lib.tg_boulder_generate(C.byref(pop), region.ctypes.data, 0.0, None, 0,
                                   C.byref(n)) == 1  # TG_ERROR_ARGUMENT
