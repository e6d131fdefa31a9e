"""Crater lists (terraingen_b200.feature_lists) against the reference's own WriteCraterList files
(tests/golden/lists/, tests/golden/list_cases.py): CSV and JSON byte for byte, and a population
drawn by tg_crater_generate written and read back."""

from __future__ import annotations

import csv
import importlib.util
import json

import numpy as np
import pytest

from conftest import GOLDEN
from terraingen_b200.feature_lists import write_crater_list

_spec = importlib.util.spec_from_file_location("list_cases", GOLDEN / "list_cases.py")
CASES = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(CASES)


@pytest.mark.parametrize("ext", ["csv", "json"])
def test_crater_list_is_the_reference_file(tmp_path, ext):
    c = CASES.columns()
    out = tmp_path / f"craters.{ext}"
    write_crater_list(out, c["x"], c["y"], c["diameter"], c["age"], c["ids"], c["manual"],
                      c["replace"])
    assert out.read_bytes() == (CASES.FIXTURES / f"craters.{ext}").read_bytes()


def test_generated_population_round_trips(tmp_path):
    from terraingen_b200.workloads import crater_population, generate_craters

    # D^-2 on [1, 100] m over a 200 m square: about 400 craters.
    pop = generate_craters(crater_population(3, 0.01, 1.0, 100.0), (0.0, 0.0, 200.0, 200.0))
    assert len(pop["x"]) > 100
    for ext in ("csv", "json"):
        out = tmp_path / f"p.{ext}"
        write_crater_list(out, pop["x"], pop["y"], pop["diameter"], pop["age"], pop["id"])
        if ext == "csv":
            rows = list(csv.DictReader(out.open()))
            got = np.array([float(r["diameter"]) for r in rows])
            ids = [int(r["id"]) for r in rows]
        else:
            rows = json.loads(out.read_text())["craters"]
            got = np.array([r["diameter"] for r in rows])
            ids = [r["id"] for r in rows]
        assert np.array_equal(got, pop["diameter"])
        assert ids == [int(i) for i in pop["id"]]
