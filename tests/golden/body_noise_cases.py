"""The SyntheticSource-on-a-sphere cases tests/golden/body_noise.npz pins: stacks of fractals of
every basis and type, blended and warped, at sites on a sphere of the Moon's radius, and the
reference CPU path's heights for each (run `python tests/golden/body_noise_cases.py` with the
reference harness built, `make -C oracle ref`)."""

from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RADIUS = 1737400.0


def cases() -> dict:
    sys.path.insert(0, str(HERE.parents[1]))
    from terraingen_b200 import GridSpec
    from terraingen_b200.layouts import fractal

    degree = 1.0 / (RADIUS * math.pi / 180.0)  # degrees per meter along a meridian
    stacks = {
        # basis (Perlin, simplex, value, Worley F1 / F2 / F2-F1, Voronoi) x type (fBm, ridged,
        # billow, hybrid), blends, a warp; 3 to 6 octaves
        "perlin_fbm": [fractal(seed=1, wavelength=500.0, amplitude=50.0, octaves=6)],
        "simplex_ridged_max": [fractal(seed=2, wavelength=300.0, amplitude=20.0, octaves=5,
                                       basis=1, type=1),
                               fractal(seed=3, wavelength=120.0, amplitude=5.0, octaves=4,
                                       basis=2, type=2, blend=1)],
        "worley_hybrid_mask": [fractal(seed=4, wavelength=200.0, amplitude=30.0, octaves=4,
                                       basis=3, type=3, offset=0.7),
                               fractal(seed=5, wavelength=150.0, amplitude=8.0, octaves=3,
                                       basis=4, blend=3),
                               fractal(seed=6, wavelength=80.0, amplitude=4.0, octaves=3,
                                       basis=5, blend=2),
                               fractal(seed=7, wavelength=60.0, amplitude=2.0, octaves=3,
                                       basis=6)],
        "warped": [fractal(seed=8, wavelength=400.0, amplitude=40.0, octaves=5,
                           warp_amplitude=60.0, warp_wavelength=700.0)],
    }
    sites = {
        # a site near the equator and one at high latitude, 1 m and 4 m cells
        "equator": GridSpec(96, 80, 10.0, 1.0, degree),
        "north": GridSpec(64, 72, -123.4, 78.0, 4.0 * degree),
    }
    return {"stacks": stacks, "sites": sites}


def main() -> int:
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H

    lib = H.reference()
    c = cases()
    out = {}
    for sname, stack in c["stacks"].items():
        for gname, grid in c["sites"].items():
            out[f"{sname}_{gname}"] = H.body_noise(lib, np.array(stack), 1000.0, RADIUS, grid)
    np.savez_compressed(HERE / "body_noise.npz", **out)
    print({k: (float(v.min()), float(v.max())) for k, v in out.items()})
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
