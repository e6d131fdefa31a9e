"""The crater-list case tests/golden/lists/ holds: the reference's WriteCraterList output for the
columns below, in CSV and JSON (run `python tests/golden/list_cases.py` with the reference harness
built, `make -C oracle ref`). The columns come from a seeded generator with edge values spliced in
(integral, huge, tiny, subnormal and signed-zero doubles; the largest and smallest ids), so the
tests rebuild them."""

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


def main() -> int:
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H

    lib = H.reference()
    FIXTURES.mkdir(exist_ok=True)
    c = columns()
    for ext, js in (("csv", 0), ("json", 1)):
        H.write_crater_list(lib, FIXTURES / f"craters.{ext}", c["x"], c["y"], c["diameter"],
                            c["age"], c["ids"], c["manual"], c["replace"], js)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
