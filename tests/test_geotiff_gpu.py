"""tg_geotiff_write (the tiles laid out, predicted and LZW-coded on the device) against the
reference's files (tests/golden/geotiff/): byte for byte with None and LZW, from host arrays and
from device tensors; Deflate (zlib on host threads) with the reference's tags and decoded data;
a 1025 x 1025 terrain at the reference's default 256-pixel tiles against the restatement; the
reference's refusals."""

from __future__ import annotations

import importlib.util

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import geotiff as O

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location("geotiff_cases", GOLDEN / "geotiff_cases.py")
CASES = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(CASES)
ALL = CASES.cases()


def _grid(bands, transform):
    h, w = bands[0].shape
    return (w, h, transform)


def _write(device, path, bands, transform, kw, on_device):
    if on_device:
        import torch

        bands = [torch.from_numpy(np.ascontiguousarray(b)).cuda() for b in bands]
    keys = None
    if "directory" in kw:
        keys = (kw["directory"], kw.get("doubles", ()), kw.get("ascii", ""))
    device.geotiff_write(path, bands, _grid(bands, transform), nodata=kw.get("nodata"),
                         geokeys=keys, compression=kw["compression"],
                         tile_size=kw["tile_size"], big_tiff=kw.get("big_tiff", False))
    return path.read_bytes()


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("name", sorted(ALL))
def test_file_is_the_reference_file(device, tmp_path, name, on_device):
    bands, transform, kw = CASES.split(ALL[name])
    want = (CASES.FIXTURES / f"{name}.tif").read_bytes()
    got = _write(device, tmp_path / "out.tif", bands, transform, kw, on_device)
    if kw["compression"] == "deflate":
        a, b = O.read(got), O.read(want)
        for tag in set(a["tags"]) | set(b["tags"]):
            if tag not in (324, 325):
                assert a["tags"][tag] == b["tags"][tag], tag
        for x, y in zip(a["bands"], b["bands"]):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    else:
        assert got == want


def test_default_tiles_of_a_terrain(device, tmp_path):
    # 1025 x 1025 cells of a smooth surface with detail, the reference's 256-pixel LZW tiles.
    rng = np.random.default_rng(11)
    y, x = np.mgrid[0:1025, 0:1025] * 0.5
    z = (300.0 * np.sin(x / 90.0) * np.cos(y / 70.0) + rng.standard_normal((1025, 1025)) * 0.05)
    z = z.astype(np.float32)
    transform = (1000.0, 0.5, 0.0, 2000.0, 0.0, -0.5)
    kw = dict(nodata=float("nan"), compression="lzw", tile_size=256)
    got = _write(device, tmp_path / "t.tif", [z], transform, kw, True)
    assert got == O.write([z], transform, **kw)


def test_refusals(device, tmp_path):
    from terraingen_b200 import TgError

    z = np.zeros((20, 20), np.float32)
    g = (20, 20, (0.0, 1.0, 0.0, 0.0, 0.0, -1.0))
    with pytest.raises(TgError, match="multiple of 16"):
        device.geotiff_write(tmp_path / "a.tif", [z], g, tile_size=24)
    with pytest.raises(KeyError):
        device.geotiff_write(tmp_path / "b.tif", [z], g, compression="packbits")
    with pytest.raises(ValueError):
        device.geotiff_write(tmp_path / "c.tif", [np.zeros((10, 20), np.float32)], g)
