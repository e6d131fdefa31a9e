"""The GeoTIFF writer's restatement (oracle/geotiff.py) against the reference's own files
(tests/golden/geotiff/, written by WriteGeoTiff through the harness; tests/golden/geotiff_cases.py):
byte for byte with None and LZW compression, the same tags and decoded data with Deflate."""

from __future__ import annotations

import importlib.util

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import geotiff as O

_spec = importlib.util.spec_from_file_location("geotiff_cases", GOLDEN / "geotiff_cases.py")
CASES = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(CASES)
ALL = CASES.cases()


def _same(a: np.ndarray, b: np.ndarray) -> bool:
    return np.array_equal(a.view(np.uint32), np.ascontiguousarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("name", sorted(ALL))
def test_restatement_is_the_reference_file(name):
    bands, transform, kw = CASES.split(ALL[name])
    want = (CASES.FIXTURES / f"{name}.tif").read_bytes()
    got = O.write(bands, transform, **kw)
    if kw["compression"] == "deflate":
        a, b = O.read(got), O.read(want)
        for tag in set(a["tags"]) | set(b["tags"]):
            if tag not in (324, 325):
                assert a["tags"][tag] == b["tags"][tag], tag
        assert all(_same(x, y) for x, y in zip(a["bands"], b["bands"]))
    else:
        assert got == want


@pytest.mark.parametrize("name", sorted(ALL))
def test_reference_file_holds_the_rasters(name):
    bands, _, kw = CASES.split(ALL[name])
    r = O.read((CASES.FIXTURES / f"{name}.tif").read_bytes())
    assert len(r["bands"]) == len(bands)
    assert all(_same(x, y) for x, y in zip(r["bands"], bands))
    assert r["big"] == kw.get("big_tiff", False)


def test_lzw_round_trip_and_table_clears():
    rng = np.random.default_rng(5)
    data = rng.integers(0, 256, 40000, dtype=np.uint8).tobytes()
    coded = O.lzw_encode(data)
    assert O.lzw_decode(coded, len(data)) == data
    # Incompressible data passes 4094 codes many times: each pass writes a Clear.
    assert len(coded) > len(data)
