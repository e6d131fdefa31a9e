"""The GeoTIFF cases the fixtures under tests/golden/geotiff/ hold: the reference's WriteGeoTiff
output for each (run `python tests/golden/geotiff_cases.py` with the reference harness built,
`make -C oracle ref`). The rasters come from seeded generators, so the tests rebuild them."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
FIXTURES = HERE / "geotiff"


def cases() -> dict:
    rng = np.random.default_rng(3)
    noisy = (rng.standard_normal((45, 70)) * 10).astype(np.float32)
    walk = np.cumsum(np.cumsum(rng.standard_normal((130, 200)), 0), 1).astype(np.float32)
    holes = walk[:100, :150].copy()
    holes[20:40, 30:70] = np.nan
    sphere = [1, 1, 0, 8, 1024, 0, 1, 2, 1025, 0, 1, 1, 2048, 0, 1, 32767, 2050, 0, 1, 32767,
              2054, 0, 1, 9102, 2056, 0, 1, 32767, 2057, 34736, 1, 0, 2058, 34736, 1, 1]
    north = (100.0, 0.5, 0.0, 200.0, 0.0, -0.5)
    return {
        # One band, north-up, NaN no-data, LZW, edge tiles padded.
        "noisy_lzw": dict(bands=[noisy], transform=north, nodata=float("nan"), compression="lzw",
                          tile_size=32),
        "noisy_none": dict(bands=[noisy], transform=north, nodata=None, compression="none",
                           tile_size=32),
        "noisy_deflate": dict(bands=[noisy], transform=north, nodata=None,
                              compression="deflate", tile_size=32),
        # 16 KiB tiles of rough data: the LZW table fills and clears within a tile.
        "walk_lzw": dict(bands=[walk], transform=(0.0, 1.0, 0.0, 0.0, 0.0, 1.0),
                         nodata=-9999.0, compression="lzw", tile_size=64),
        # Holes of NaN, sphere keys (degrees on the Moon), a value no-data.
        "holes_sphere": dict(bands=[holes], transform=(-10.0, 0.01, 0.0, 5.0, 0.0, -0.01),
                             nodata=-32768.0, directory=sphere, doubles=[1737400.0, 1737400.0],
                             compression="lzw", tile_size=48),
        # Two bands, a rotated PixelIsPoint transform, ASCII params, BigTIFF, 16-pixel tiles.
        "bands_rotated_big": dict(bands=[noisy, noisy * 2.0], transform=(1.0, 0.5, 0.1, 2.0, 0.2,
                                                                        -0.5),
                                  nodata=None, directory=[1, 1, 0, 2, 1024, 0, 1, 2, 1025, 0, 1, 2],
                                  doubles=[1.5], ascii="moon|", compression="lzw", tile_size=16,
                                  big_tiff=True),
    }


def split(case: dict):
    """(bands, transform, the writer's keyword arguments) of a case."""
    kw = dict(case)
    return kw.pop("bands"), kw.pop("transform"), kw


def main() -> int:
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle import harness as H

    lib = H.reference()
    FIXTURES.mkdir(exist_ok=True)
    for name, case in cases().items():
        bands, transform, kw = split(case)
        H.write_geotiff(lib, FIXTURES / f"{name}.tif", bands, transform, **kw)
        print(name, (FIXTURES / f"{name}.tif").stat().st_size)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
