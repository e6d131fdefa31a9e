"""The list cases tests/golden/lists/ holds: the reference's WriteCraterList and WriteBoulderList
output for the columns below, in CSV and JSON, and an empty boulder list (run
`python tests/golden/list_cases.py` with the reference harness built, `make -C oracle ref`). The
columns come from seeded generators with edge values spliced in (integral, huge, tiny, subnormal
and signed-zero doubles, doubles in [1e15, 1e16) where JSON changes to an exponent, infinities and
NaNs of both signs, unset grounds; the largest and smallest ids), so the tests rebuild them."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
FIXTURES = HERE / "lists"


def columns() -> dict:
    rng = np.random.default_rng(4)
    n = 40
    x = rng.uniform(-1e6, 1e6, n)
    y = rng.uniform(-1e3, 1e3, n)
    d = np.exp(rng.uniform(0, 6, n))
    age = rng.uniform(0, 4, n)
    x[0], x[1], x[2], x[3], x[8] = 1.0, 1e20, 1e-7, -0.0, 2.5e-320
    y[4], d[5], age[6], age[7] = 123456789.0, 0.1, 0.0, 1e16
    ids = rng.integers(0, 2**63, n, dtype=np.uint64)
    ids[0], ids[1] = 2**64 - 1, 0
    manual = rng.integers(0, 2, n).astype(np.uint8)
    replace = rng.integers(0, 2, n).astype(np.uint8)
    return dict(x=x, y=y, diameter=d, age=age, ids=ids, manual=manual, replace=replace)


def boulder_columns(n: int = 40) -> dict:
    """A boulder list's columns as the harness takes them (angles in radians, NaN grounds
    unset)."""
    rng = np.random.default_rng(5)
    c = dict(x=rng.uniform(-1e5, 1e5, n), y=rng.uniform(-1e5, 1e5, n),
             diameter=np.exp(rng.uniform(-1.6, 1.1, n)), burial=rng.uniform(0, 0.6, n),
             yaw=rng.uniform(-np.pi, np.pi, n), lean=rng.uniform(0, 0.3, n),
             tilt=rng.uniform(0, 0.4, n), tilt_azimuth=rng.uniform(-np.pi, np.pi, n),
             wear=rng.uniform(0, 1, n), ground=rng.uniform(-2000, 2000, n))
    c["height"] = c["diameter"] * rng.uniform(0.3, 0.9, n)
    if n:
        c["x"][:6] = [1e15, 1234567890123456.2, -9999999999999998.0, 1e16, 999999999999999.9,
                      2.5e-320]
        c["y"][:4] = [-0.0, 1e-4, 1e-5, 123456789.0]
        c["ground"][::3] = np.nan
        c["ground"][1], c["ground"][2] = 0.0, -0.0
        c["yaw"][0], c["yaw"][1], c["lean"][2] = np.inf, -np.inf, np.pi
        c["wear"][0], c["wear"][1] = np.nan, np.copysign(np.nan, -1.0)
    c["id"] = rng.integers(0, 2**63, n, dtype=np.uint64)
    c["parent"] = np.where(rng.uniform(size=n) < 0.3, c["id"] ^ np.uint64(7), np.uint64(0))
    c["piece"] = rng.integers(0, 6, n).astype(np.uint32)
    c["rest"] = rng.integers(0, 3, n).astype(np.uint8)
    c["model"] = (rng.uniform(size=n) < 0.2).astype(np.uint8)
    if n:
        c["id"][0], c["parent"][1], c["piece"][2] = 2**64 - 1, 2**64 - 1, 2**32 - 1
    return c


def main() -> int:
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H

    lib = H.reference()
    FIXTURES.mkdir(exist_ok=True)
    c = columns()
    for ext, js in (("csv", 0), ("json", 1)):
        H.write_crater_list(lib, FIXTURES / f"craters.{ext}", c["x"], c["y"], c["diameter"],
                            c["age"], c["ids"], c["manual"], c["replace"], js)
        H.write_boulder_list(lib, FIXTURES / f"boulders.{ext}", boulder_columns(), js)
        H.write_boulder_list(lib, FIXTURES / f"boulders_empty.{ext}", boulder_columns(0), js)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
