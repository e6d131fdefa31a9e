"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run here, where the reference sources are, after `make -C oracle`:

    python tests/golden/make_fixtures.py

Each fixture holds the inputs the reference hands its GPU backend (captured through the drop-in
device, oracle/ref_harness.cpp) and the reference CPU path's heights for the same scene, so the
GPU tests need nothing from the reference at run time.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import harness as H  # noqa: E402
from terraingen_b200 import GridSpec, centered, layouts as L  # noqa: E402

OUT = Path(__file__).resolve().parent


def noise_fixtures() -> None:
    ref = H.reference()
    cases = {}
    # The synthetic source of the 4097^2 terrain (8-octave Perlin fBm, 512 m, 5 m), a window.
    g = centered(96, 80, 0.5, 123.25, -37.5)
    f = L.fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)
    cases["fbm"] = (g, np.array([f]), 0.0)
    # The DEM source (12 octaves, 20 km, 2000 m) at 5 m.
    g = centered(64, 64, 5.0, -2500.0, 4000.0)
    f = L.fractal(seed=3, wavelength=20000.0, amplitude=2000.0, octaves=12)
    cases["dem"] = (g, np.array([f]), 100.0)
    # A stack with every basis, type and blend, a warp and a disabled fractal.
    g = centered(48, 40, 2.0, 900.0, 700.0)
    stack = np.array([
        L.fractal(seed=1, wavelength=300.0, amplitude=20.0, octaves=5),
        L.fractal(seed=2, wavelength=120.0, amplitude=6.0, octaves=3, basis=1, type=1, blend=0),
        L.fractal(seed=3, wavelength=90.0, amplitude=4.0, octaves=4, basis=2, type=2, blend=1),
        L.fractal(seed=4, wavelength=70.0, amplitude=5.0, octaves=3, basis=3, type=3, blend=2,
                  offset=0.7),
        L.fractal(seed=5, wavelength=60.0, amplitude=3.0, octaves=2, basis=5, blend=0,
                  warp_amplitude=25.0, warp_wavelength=200.0),
        L.fractal(seed=6, wavelength=50.0, amplitude=2.0, octaves=2, basis=6, blend=3),
        L.fractal(seed=8, wavelength=40.0, amplitude=9.0, octaves=2, basis=4, enabled=False),
        L.fractal(seed=9, wavelength=33.0, amplitude=1.5, octaves=6, type=1, offset=1.2),
    ])
    cases["stack"] = (g, stack, -5.0)
    # Far from the origin (1.2e5 m): float positions as the reference narrows them.
    g = centered(40, 40, 1.0, 120000.0, -80000.0)
    cases["far"] = (g, np.array([L.fractal(seed=11, wavelength=800.0, amplitude=40.0)]), 0.0)
    arrays = {}
    for name, (grid, fractals, elevation) in cases.items():
        scene = H.make_scene(grid, source_fractals=fractals, elevation=elevation)
        heights, _ = H.evaluate(ref, scene, 0, 1)
        arrays[f"{name}_grid"] = np.array([grid.width, grid.height, grid.x0, grid.y0, grid.pixel])
        arrays[f"{name}_fractals"] = fractals.view(np.uint8)
        arrays[f"{name}_elevation"] = np.float32(elevation)
        arrays[f"{name}_heights"] = heights
    # A noise layer over a synthetic source: the layer runs through RunKernel (captured).
    g = centered(70, 50, 1.0, 10.0, 20.0)
    src = np.array([L.fractal(seed=21, wavelength=400.0, amplitude=30.0, octaves=6)])
    lay = np.array([L.fractal(seed=22, wavelength=60.0, amplitude=2.0, octaves=4),
                    L.fractal(seed=23, wavelength=25.0, amplitude=0.5, octaves=3, basis=1)])
    scene = H.make_scene(g, source_fractals=src, layer_fractals=lay)
    heights, _ = H.evaluate(ref, scene, 0, 1)
    cap = H.capture()
    H.evaluate(cap, scene, 1, 1)
    (call,) = H.captured(cap)
    assert call["kind"] == 1
    for k in ("kernel", "xs", "ys", "heights"):
        arrays[f"layer_{k}"] = call[k]
    arrays["layer_expected"] = heights
    np.savez_compressed(OUT / "noise.npz", **arrays)


CRATER_SCENES = {
    # The 257^2, 1 m crater terrain: Fassett-Thomson, irregular outlines (the default apply).
    "config1": (centered(257, 257, 1.0), H.config1_craters()),
    # Martin-Parkes-Dunstan, plain options, off-center grid.
    "mpd": (centered(160, 144, 0.5, 40.0, -25.0),
            dict(seed=5, sfdCoefficient=4e-2, minDiameter=1.0, maxDiameter=40.0, profile=1,
                 applyPreset=1)),
    # Complex craters (lowered transition) with peaks and terraces, rim smoothing.
    "complex": (centered(192, 192, 2.0),
                dict(seed=9, sfdCoefficient=0.6, minDiameter=8.0, maxDiameter=300.0, profile=2,
                     transitionDiameter=60.0, terraceOnset=80.0, terraceFull=200.0,
                     rimSigma=0.08)),
    # The reference's default crater models (diffused MPD profiles, matched diffusion).
    "diffused": (centered(160, 160, 2.0, 300.0, 300.0),
                 dict(seed=3, sfdCoefficient=0.2, minDiameter=10.0, maxDiameter=120.0, profile=3)),
    # Crater noise and texture (wall streaks, ejecta).
    "textured": (centered(128, 128, 1.0),
                 dict(seed=4, sfdCoefficient=3e-2, minDiameter=4.0, maxDiameter=60.0, profile=1,
                      noiseAmplitude=0.02, rimNoiseAmplitude=0.01, wallStreaks=0.01,
                      ejecta=0.5)),
}


def crater_fixtures() -> None:
    ref = H.reference()
    cap = H.capture()
    arrays = {}
    for name, (grid, fields) in CRATER_SCENES.items():
        scene = H.make_scene(grid, craters=fields)
        heights, _ = H.evaluate(ref, scene, 0, 1)
        H.evaluate(cap, scene, 1, 1)
        calls = [c for c in H.captured(cap) if c["kind"] == 2]
        assert len(calls) == 1, (name, len(calls))
        call = calls[0]
        arrays[f"{name}_grid"] = np.array([grid.width, grid.height, grid.x0, grid.y0,
                                           grid.pixel])
        for k in H.CRATER_FIELDS:
            arrays[f"{name}_{k}"] = call[k]
        arrays[f"{name}_expected"] = heights
        print(name, len(call["records"]) // 144, "craters",
              len(call["data"]) // 4, "data floats", float(np.abs(heights).max()))
    np.savez_compressed(OUT / "craters.npz", **arrays)


def boulder_fixtures() -> None:
    """Boulders drawn as domes over an fBm source: the boulders the reference's layer draws, the
    heights beneath them and the reference heights with them."""
    ref = H.reference()
    arrays = {}
    cases = {
        # 0.5 m cells, sizes D^-2.5 on [0.2, 3] m, heights 0.5 D (the 4097^2 terrain's boulders).
        "dense": (centered(200, 160, 0.5, 10.0, 5.0), dict(boulderCoefficient=0.5)),
        # 0.25 m cells: more boulders resolved, off-center.
        "fine": (centered(128, 128, 0.25, -300.0, 120.0),
                 dict(boulderSeed=4, boulderCoefficient=0.3, heightRatio=0.4)),
    }
    for name, (grid, fields) in cases.items():
        src = np.array([L.fractal(seed=7, wavelength=64.0, amplitude=1.5, octaves=5)])
        scene = H.make_scene(grid, source_fractals=src, boulders=fields)
        arrays[f"{name}_grid"] = np.array([grid.width, grid.height, grid.x0, grid.y0, grid.pixel])
        arrays[f"{name}_boulders"] = H.boulders(ref, scene)
        arrays[f"{name}_base"] = H.below_boulders(ref, scene, 1)
        arrays[f"{name}_expected"], _ = H.evaluate(ref, scene, 0, 1)
        print(name, len(arrays[f"{name}_boulders"]), "boulders")
    # Heights and burial drawn between bounds (the pose streams), without ground.
    grid = centered(180, 150, 0.5, -40.0, 75.0)
    scene = H.make_scene(grid, boulders=dict(boulderSeed=9, boulderCoefficient=0.4))
    pose = (0.3, 0.7, 0.1, 0.4)
    arrays["posed_grid"] = np.array([grid.width, grid.height, grid.x0, grid.y0, grid.pixel])
    arrays["posed_pose"] = np.array(pose)
    arrays["posed_boulders"] = H.boulders_posed(ref, scene, pose)
    print("posed", len(arrays["posed_boulders"]), "boulders")
    np.savez_compressed(OUT / "boulders.npz", **arrays)


def ds_fixtures() -> None:
    """Diamond-square refinement of seeded DEMs by the reference's DiamondSquareUpsampler."""
    ref = H.reference()
    rs = H.restate()
    arrays = {}
    cases = {
        # 65 x 65 posts at 5 m (a 12-octave fBm DEM, 20 km / 2000 m), read at 1 m: 3 levels.
        "dem5m": (centered(65, 65, 5.0), centered(301, 301, 1.0, 3.25, -1.75), 2.2, 1.5, 7),
        # Posts at 4 m read at 0.5 m off-center: exactly 3 levels, nodes on cell centers.
        "exact": (centered(48, 40, 4.0, 100.0, 60.0), centered(240, 200, 0.5, 90.0, 70.0), 2.5,
                  0.8, 3),
        # Ten-fold, as the 20481^2 refinement (4 levels), on a small window.
        "tenfold": (centered(41, 41, 5.0), centered(351, 351, 0.5, -10.0, 5.0), 2.2, 2.0, 11),
        # Catmull-Rom (DiamondSquareInterp::CatmullRom): spline midpoints and the cubic read.
        "dem5m_cr": (centered(65, 65, 5.0), centered(301, 301, 1.0, 3.25, -1.75), 2.2, 1.5, 7),
        "tenfold_cr": (centered(41, 41, 5.0), centered(351, 351, 0.5, -10.0, 5.0), 2.2, 2.0, 11),
    }
    for name, (pg, grid, fd, scale, seed) in cases.items():
        interp = 1 if name.endswith("_cr") else 0
        posts = np.zeros((pg.height, pg.width), np.float32)
        rs.rs_fbm_grid_f32(pg.width, pg.height, pg.x0, pg.y0, pg.pixel, 3, 20000.0, 2000.0, 12,
                           2.0, 0.5, 0.0, posts.ctypes.data)
        heights, _ = H.diamond_square(ref, posts, pg, grid, fd, scale, seed, interp, 1)
        assert not np.isnan(heights).any(), name
        arrays[f"{name}_posts"] = posts
        arrays[f"{name}_post_grid"] = np.array([pg.width, pg.height, pg.x0, pg.y0, pg.pixel])
        arrays[f"{name}_grid"] = np.array([grid.width, grid.height, grid.x0, grid.y0, grid.pixel])
        arrays[f"{name}_options"] = np.array([fd, scale, seed, interp], np.float64)
        arrays[f"{name}_expected"] = heights
        print(name, heights.shape, float(heights.std()))
    np.savez_compressed(OUT / "ds.npz", **arrays)


def _seam_rasters(grid, seed: int, hole) -> tuple[np.ndarray, np.ndarray]:
    """An fBm `earlier` raster with NaN where `hole(x, y)` holds, and a `later` one offset from it
    by a smooth bias of a few meters (a coarser DEM that disagrees with the patch)."""
    rs = H.restate()
    earlier = np.zeros((grid.height, grid.width), np.float32)
    rs.rs_fbm_grid_f32(grid.width, grid.height, grid.x0, grid.y0, grid.pixel, seed, 300.0, 25.0,
                       6, 2.0, 0.5, 0.0, earlier.ctypes.data)
    cols = np.arange(grid.width) + 0.5
    rows = np.arange(grid.height) + 0.5
    x = grid.x0 + cols[None, :] * grid.pixel
    y = grid.y0 - rows[:, None] * grid.pixel
    u = (x - grid.x0) / (grid.width * grid.pixel)
    v = (grid.y0 - y) / (grid.height * grid.pixel)
    bias = 2.5 + 1.5 * u - 2.0 * v + 0.8 * np.sin(6.0 * u + 1.0) * np.cos(4.0 * v)
    later = (earlier - bias).astype(np.float32)
    earlier = np.where(hole(x, y), np.float32(np.nan), earlier).astype(np.float32)
    return earlier, later


SEAM_SCENES = {
    # A hole inside a 200 x 150 m patch at 1 m (an ellipse with a notch): the three modes.
    "hole": (centered(200, 150, 1.0, 500.0, -300.0),
             lambda x, y: (((x - 490.0) / 45.0) ** 2 + ((y + 310.0) / 30.0) ** 2 < 1.0)
             | ((np.abs(x - 540.0) < 6.0) & (np.abs(y + 300.0) < 20.0)), 3),
    # One of 2 x 2 patches at 2 m: the earlier source covers the top-left quadrant only, so the
    # gap is an L reaching the raster's edges (the seam between patches).
    "patch": (centered(160, 140, 2.0, -1200.0, 800.0),
              lambda x, y: (x > -1200.0 + 4.0) | (y < 800.0 - 10.0), 5),
}
SEAM_MODES = {
    "hole": [("feather", 1, 10.0, 0.0), ("height", 2, 0.0, 6.0), ("slope", 3, 0.0, 6.0)],
    "patch": [("feather", 1, 16.0, 0.0), ("height", 2, 0.0, 8.0), ("slope", 3, 0.0, 8.0)],
}


def seam_fixtures() -> None:
    """The reference's seam fields (BuildSeamField) from its own lattice samples, and the chain's
    heights (SourceChain::FillGridGaps) on the rasters' grid and on a finer window."""
    ref = H.reference()
    arrays = {}
    nan = np.float32(np.nan)
    for scene, (grid, hole, seed) in SEAM_SCENES.items():
        earlier, later = _seam_rasters(grid, seed, hole)
        t = grid.transform()
        arrays[f"{scene}_grid"] = np.array([grid.width, grid.height, grid.x0, grid.y0,
                                            grid.pixel])
        arrays[f"{scene}_earlier"] = earlier
        arrays[f"{scene}_later"] = later
        # A finer window across the gap's edge, read from each source alone: the earlier source
        # (NaN where it has no data) and the later one.
        fine = centered(150, 110, 0.5 * grid.pixel, grid.x0 + 0.55 * grid.width * grid.pixel,
                        grid.y0 - 0.5 * grid.height * grid.pixel)
        arrays[f"{scene}_fine_grid"] = np.array([fine.width, fine.height, fine.x0, fine.y0,
                                                 fine.pixel])
        none_later = np.full_like(later, nan)
        none_earlier = np.full_like(earlier, nan)
        arrays[f"{scene}_fine_earlier"] = H.chain(ref, earlier, none_later, t, 0, 1.0, 1.0, fine)
        arrays[f"{scene}_fine_later"] = H.chain(ref, none_earlier, later, t, 0, 1.0, 1.0, fine)
        for name, mode, width, decay in SEAM_MODES[scene]:
            s = H.seam(ref, earlier, later, t, mode, width or 50.0, decay or 50.0)
            key = f"{scene}_{name}"
            arrays[f"{key}_options"] = np.array([mode, width or 50.0, decay or 50.0])
            arrays[f"{key}_lattice"] = np.array([s["width"], s["height"], *s["transform"]])
            arrays[f"{key}_data"] = s["data"]
            arrays[f"{key}_difference"] = s["difference"]
            arrays[f"{key}_field"] = s["field"]
            arrays[f"{key}_ms"] = np.float64(s["ms"])
            arrays[f"{key}_chain"] = H.chain(ref, earlier, later, t, mode, width or 50.0,
                                             decay or 50.0, grid)
            arrays[f"{key}_fine_chain"] = H.chain(ref, earlier, later, t, mode, width or 50.0,
                                                  decay or 50.0, fine)
            print(key, s["width"], "x", s["height"], "posts,",
                  int(np.count_nonzero(s["field"])), "set,", f"{s['ms']:.1f} ms")
    np.savez_compressed(OUT / "seams.npz", **arrays)


def chain_fixture() -> None:
    """Four raster patches (2 x 2 windows of a grid with a 16-cell overlap, each its own fBm and a
    datum offset) chained by the reference's SourceChain with each seam mode."""
    ref = H.reference()
    rs = H.restate()
    grid = centered(300, 260, 1.0, 2000.0, -500.0)
    arrays = {"grid": np.array([grid.width, grid.height, grid.x0, grid.y0, grid.pixel])}
    windows = []
    for r0, r1 in ((0, 138), (122, 260)):
        for c0, c1 in ((0, 158), (142, 300)):
            windows.append((c0, r0, c1 - c0, r1 - r0))
    patches, grids = [], []
    for k, (c0, r0, w, h) in enumerate(windows):
        g = GridSpec(w, h, grid.x0 + c0 * grid.pixel, grid.y0 - r0 * grid.pixel, grid.pixel)
        p = np.zeros((h, w), np.float32)
        rs.rs_fbm_grid_f32(w, h, g.x0, g.y0, g.pixel, 40 + k, 200.0, 12.0, 5, 2.0, 0.5,
                           0.6 * k, p.ctypes.data)
        patches.append(p)
        grids.append(g)
        arrays[f"patch{k}"] = p
    arrays["windows"] = np.array(windows)
    for name, mode, width, decay in (("feather", 1, 10.0, 50.0), ("height", 2, 50.0, 4.0),
                                     ("slope", 3, 50.0, 4.0)):
        out = H.patch_chain(ref, patches, grids, mode, width, decay, grid)
        assert not np.isnan(out).any(), name
        arrays[f"{name}_options"] = np.array([mode, width, decay])
        arrays[f"{name}_heights"] = out
        print("chain", name, float(out.min()), float(out.max()))
    np.savez_compressed(OUT / "chain.npz", **arrays)


DATUM_SCENE = (centered(200, 200, 1.0, 40.0, -30.0),
               dict(seed=3, sfdCoefficient=0.08, minDiameter=3.0, maxDiameter=60.0, profile=0,
                    applyPreset=1, datum=1, interiorReplacement=0.5))


def datum_fixture() -> None:
    """Crater datums fitted as planes: the tg_crater_datums call the reference makes (captured)
    with the lattice after the reference's own KernelDatumRelief, and the scene's CPU heights."""
    ref = H.reference()
    cap = H.capture()
    grid, fields = DATUM_SCENE
    src = np.array([L.fractal(seed=5, wavelength=150.0, amplitude=8.0, octaves=5)])
    scene = H.make_scene(grid, source_fractals=src, craters=fields)
    arrays = {"grid": np.array([grid.width, grid.height, grid.x0, grid.y0, grid.pixel]),
              "source": src.view(np.uint8)}
    arrays["expected"], _ = H.evaluate(ref, scene, 0, 1)
    H.evaluate(cap, scene, 1, 1)
    calls = [c for c in H.captured(cap) if c["kind"] == 3]
    assert len(calls) == 1, len(calls)
    call = calls[0]
    for k in H.DATUM_FIELDS:
        arrays[f"call_{k}"] = call[k]
    arrays["call_shape"] = np.array([call["width"], call["rows"], call["first_row"]])
    arrays["relief"] = H.datum_relief(ref, call)
    print("datums", call["rows"], "fitted,", len(call["records"]) // 144, "records")
    np.savez_compressed(OUT / "datums.npz", **arrays)


def population_fixture() -> None:
    """The config-1 crater population (centers, diameters, ages, ids): bit-exact targets."""
    ref = H.reference()
    scene = H.make_scene(centered(257, 257, 1.0), craters=H.config1_craters())
    pop = H.craters(ref, scene, (-128.5, -128.5, 128.5, 128.5), 1.0)
    np.savez_compressed(OUT / "population.npz", **pop)


if __name__ == "__main__":
    H.build("ref")
    H.build("capture")
    noise_fixtures()
    crater_fixtures()
    boulder_fixtures()
    ds_fixtures()
    population_fixture()
    seam_fixtures()
    chain_fixture()
    datum_fixture()
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)
