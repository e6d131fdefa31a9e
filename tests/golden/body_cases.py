"""The body (sphere) crater scene tests/golden/body.npz pins: a 129 x 129 site of 1 m cells at
longitude 10, latitude 20 on a sphere of the Moon's radius with the first configuration's
craters, and the reference CPU path's heights for it (run `python tests/golden/body_cases.py`
with the reference harness built, `make -C oracle ref`)."""

from __future__ import annotations

import ctypes as C
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RADIUS = 1737400.0
SIDE = 129


def scene():
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H
    from terraingen_b200 import GridSpec

    degree = 1.0 / (RADIUS * math.pi / 180.0)  # degrees per meter along a meridian
    s = H.make_scene(GridSpec(SIDE, SIDE, 10.0, 20.0, degree), craters=H.config1_craters())
    s.bodyRadius = RADIUS
    return s


def main() -> int:
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H

    lib = H.reference()
    out = np.zeros(SIDE * SIDE, np.float32)
    ms = C.c_double()
    if lib.tgref_evaluate(C.byref(scene()), 0, 1, out.ctypes.data, C.byref(ms)) != 0:
        raise RuntimeError(lib.tgref_error().decode())
    np.savez_compressed(HERE / "body.npz", expected=out.reshape(SIDE, SIDE))
    print("craters touch", np.count_nonzero(out), "cells; max", float(np.abs(out).max()))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
