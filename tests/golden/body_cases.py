"""The body (sphere) crater scene tests/golden/body.npz pins: a 129 x 129 site of 1 m cells at
longitude 10, latitude 20 on a sphere of the Moon's radius with the first configuration's
craters, plain and with plane datums, and the reference CPU path's heights for each (run `python tests/golden/body_cases.py`
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


def scene(datum: int = 0):
    """The site; with `datum` 1 the craters cut planes fitted on the body (CraterDatum::Plane),
    which the reference fits with its body datum kernel."""
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H
    from terraingen_b200 import GridSpec

    degree = 1.0 / (RADIUS * math.pi / 180.0)  # degrees per meter along a meridian
    craters = dict(H.config1_craters())
    if datum:
        craters.update(datum=datum, interiorReplacement=0.5)
    s = H.make_scene(GridSpec(SIDE, SIDE, 10.0, 20.0, degree), craters=craters)
    s.bodyRadius = RADIUS
    return s


def main() -> int:
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H

    lib = H.reference()
    outs = {}
    for name, datum in (("expected", 0), ("datum_expected", 1)):
        out = np.zeros(SIDE * SIDE, np.float32)
        ms = C.c_double()
        if lib.tgref_evaluate(C.byref(scene(datum)), 0, 1, out.ctypes.data, C.byref(ms)) != 0:
            raise RuntimeError(lib.tgref_error().decode())
        outs[name] = out.reshape(SIDE, SIDE)
        print(name, np.count_nonzero(out), "cells touched; max", float(np.abs(out).max()))
    np.savez_compressed(HERE / "body.npz", **outs)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
