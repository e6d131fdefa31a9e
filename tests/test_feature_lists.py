"""Crater and boulder lists (terraingen_b200.feature_lists) against the reference's own
WriteCraterList and WriteBoulderList files (tests/golden/lists/, tests/golden/list_cases.py): CSV
and JSON byte for byte, an empty boulder list, and a population drawn by tg_crater_generate
written and read back."""

from __future__ import annotations

import csv
import importlib.util
import json

import numpy as np
import pytest

from conftest import GOLDEN
from terraingen_b200.feature_lists import write_boulder_list, write_crater_list

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


@pytest.mark.parametrize("ext", ["csv", "json"])
@pytest.mark.parametrize("n", [40, 0])
def test_boulder_list_is_the_reference_file(tmp_path, ext, n):
    c = CASES.boulder_columns(n)
    out = tmp_path / f"boulders.{ext}"
    write_boulder_list(out, c["x"], c["y"], c["diameter"], c["height"], burial=c["burial"],
                       yaw=c["yaw"], lean=c["lean"], ids=c["id"], ground=c["ground"],
                       model=c["model"], wear=c["wear"], parent=c["parent"], piece=c["piece"],
                       rest=c["rest"], tilt=c["tilt"], tilt_azimuth=c["tilt_azimuth"])
    name = "boulders" if n else "boulders_empty"
    assert out.read_bytes() == (CASES.FIXTURES / f"{name}.{ext}").read_bytes()


def test_boulder_list_defaults_and_json_reads_back(tmp_path):
    x, y = np.array([1.5, -2.0]), np.array([3.0, 1e15])
    out = tmp_path / "b.json"
    write_boulder_list(out, x, y, [1.0, 2.0], [0.5, 1.0])
    rows = json.loads(out.read_text())["boulders"]
    assert [r["y"] for r in rows] == [3.0, 1e15]
    assert all(r["ground"] is None and r["rest"] == 0 and r["model"] is False for r in rows)
    with pytest.raises(ValueError):
        write_boulder_list(tmp_path / "bad.csv", x, y, [1.0], [0.5, 1.0])


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
