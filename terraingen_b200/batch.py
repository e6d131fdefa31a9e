"""The batched form (tg_batch_* in include/tgb200.h): many tiles of one layer stack evaluated in
one persistent launch replayed from a CUDA graph, with an autotuner over kernel shapes.

`TileSet` holds a batch's host inputs (tile grids and output layout, the source fractal, the crater
kernel and every tile's records, the boulders); `Batch` loads it onto a device and evaluates it
into a host array or a torch CUDA tensor.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .device import Device, GridSpec, _stream
from .layouts import CRATER_RECORD, CRATER_SHAPE_KERNEL

TILE = np.dtype([("width", "<u4"), ("height", "<u4"), ("origin_x", "<f8"), ("pixel_width", "<f8"),
                 ("row_rotation", "<f8"), ("origin_y", "<f8"), ("col_rotation", "<f8"),
                 ("pixel_height", "<f8"), ("height_offset", "<u8"), ("pitch", "<u4"),
                 ("crater_begin", "<u4"), ("crater_count", "<u4"), ("data_begin", "<u4"),
                 ("boulder_begin", "<u4"), ("boulder_count", "<u4"), ("boulder_width", "<f8")])
assert TILE.itemsize == C.sizeof(N.Tile)
POINT_SET = np.dtype([("point_begin", "<u4"), ("point_count", "<u4"), ("height_offset", "<u8"),
                      ("crater_begin", "<u4"), ("crater_count", "<u4"), ("data_begin", "<u4"),
                      ("boulder_begin", "<u4"), ("boulder_count", "<u4"), ("reserved", "<u4"),
                      ("boulder_width", "<f8")])
assert POINT_SET.itemsize == C.sizeof(N.PointSet)


@dataclass
class TileSet:
    """A batch's inputs. Tile i's cells are out[offset_i + row * pitch_i + col]."""

    tiles: np.ndarray                  # TILE records
    fractals: np.ndarray               # FRACTAL records (at most one enabled)
    elevation: float
    crater_kernel: np.ndarray          # one CRATER_SHAPE_KERNEL
    crater_records: np.ndarray         # CRATER_RECORD, tile by tile
    crater_data: np.ndarray            # float32, tile by tile
    crater_footprints: np.ndarray      # float64 [3 * records]
    boulders: np.ndarray               # float64 [n, 5]
    grids: list = field(default_factory=list)  # GridSpec per tile
    point_sets: np.ndarray = field(default_factory=lambda: np.zeros(0, POINT_SET))
    points: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))  # float64 (x, y)

    @property
    def output_floats(self) -> int:
        t, p = self.tiles, self.point_sets
        ends = [0]
        if len(t):
            ends.append(int((t["height_offset"] + (t["height"].astype(np.int64) - 1) * t["pitch"]
                             + t["width"]).max()))
        if len(p):
            ends.append(int((p["height_offset"] + p["point_count"]).max()))
        return max(ends)

    @property
    def cells(self) -> int:
        return int((self.tiles["width"].astype(np.int64) * self.tiles["height"]).sum() +
                   self.point_sets["point_count"].astype(np.int64).sum())

    def input_bytes(self) -> int:
        return (self.tiles.nbytes + self.crater_records.nbytes + self.crater_data.nbytes +
                self.crater_footprints.nbytes + self.boulders.nbytes + self.point_sets.nbytes +
                self.points.nbytes)

    def point_view(self, out: np.ndarray, i: int) -> np.ndarray:
        """Point set i's heights."""
        p = self.point_sets[i]
        return out[int(p["height_offset"]):int(p["height_offset"]) + int(p["point_count"])]

    def tile_view(self, out: np.ndarray, i: int) -> np.ndarray:
        """Tile i's heights as a (height, width) view of the output array."""
        t = self.tiles[i]
        off, pitch, w, h = int(t["height_offset"]), int(t["pitch"]), int(t["width"]), int(t["height"])
        flat = out[off:off + (h - 1) * pitch + w]
        return np.lib.stride_tricks.as_strided(flat, shape=(h, w),
                                               strides=(pitch * flat.itemsize, flat.itemsize))

    def native(self) -> N.BatchInput:
        self._keep = [np.ascontiguousarray(a) for a in (
            self.tiles, self.fractals, self.crater_kernel, self.crater_records, self.crater_data,
            self.crater_footprints, self.boulders, self.point_sets,
            np.asarray(self.points, np.float64).reshape(-1, 2))]
        tiles, fractals, kernel, records, data, footprints, boulders, sets, points = self._keep
        if sets.dtype != POINT_SET:
            raise TypeError("point sets must use the POINT_SET layout")
        if records.dtype != CRATER_RECORD or kernel.dtype != CRATER_SHAPE_KERNEL:
            raise TypeError("crater records and kernel must use the std430 layouts")
        if boulders.size and (boulders.dtype != np.float64 or boulders.shape[-1] != 5):
            raise TypeError("boulders are [n, 5] float64")
        return N.BatchInput(
            tiles.ctypes.data, len(tiles), fractals.ctypes.data, len(fractals),
            float(self.elevation), kernel.ctypes.data, records.ctypes.data, len(records),
            data.ctypes.data, len(data), footprints.ctypes.data if footprints.size else None,
            boulders.ctypes.data if boulders.size else None, len(boulders),
            sets.ctypes.data if len(sets) else None, len(sets),
            points.ctypes.data if len(points) else None, len(points))


def layout(grids: list[GridSpec], align: int = 4) -> tuple[np.ndarray, np.ndarray]:
    """(height_offset, pitch) per tile for tiles stored back to back, rows padded to `align`
    floats so each row starts on a 16-byte boundary."""
    pitch = np.array([(g.width + align - 1) // align * align for g in grids], np.uint32)
    sizes = np.array([p * g.height for p, g in zip(pitch, grids)], np.uint64)
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    return offsets, pitch


class Batch:
    """tg_batch: load a TileSet, evaluate it (graph replay), tune its kernel shape."""

    def __init__(self, device: Device):
        self._device = device
        self._lib = N.library()
        handle = C.c_void_p()
        N.check(self._lib.tg_batch_create(device._handle, C.byref(handle)))
        self._handle = handle
        self.tileset: TileSet | None = None

    def close(self) -> None:
        if self._handle:
            self._lib.tg_batch_destroy(self._handle)
            self._handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, tileset: TileSet) -> None:
        native = tileset.native()
        N.check(self._lib.tg_batch_load(self._handle, C.byref(native)))
        self.tileset = tileset

    def evaluate(self, out) -> None:
        """Evaluates into `out`: a float32 numpy array (host) or a torch CUDA float32 tensor of at
        least output_floats elements."""
        if type(out).__module__.startswith("torch"):
            memory = N.TG_MEMORY_DEVICE
            n = out.numel()
            p = C.c_void_p(out.data_ptr())
        else:
            if out.dtype != np.float32 or not out.flags.c_contiguous:
                raise TypeError("out must be a contiguous float32 array")
            memory = N.TG_MEMORY_HOST
            n = out.size
            p = C.c_void_p(out.ctypes.data)
        N.check(self._lib.tg_batch_evaluate(self._handle, p, n, memory, _stream(memory)))

    def run(self, tileset: TileSet, out) -> None:
        self.load(tileset)
        self.evaluate(out)

    def tune(self, trials: int = 3) -> list[float]:
        count = self._lib.tg_batch_variant_count()
        ms = (C.c_float * count)()
        N.check(self._lib.tg_batch_tune(self._handle, trials, ms))
        return list(ms)

    def set_variant(self, index: int) -> None:
        N.check(self._lib.tg_batch_set_variant(self._handle, index))

    @staticmethod
    def variants() -> list[tuple[int, int, int]]:
        lib = N.library()
        out = []
        for i in range(lib.tg_batch_variant_count()):
            w, h, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
            N.check(lib.tg_batch_variant(i, C.byref(w), C.byref(h), C.byref(c)))
            out.append((w.value, h.value, c.value))
        return out

    def stats(self) -> dict:
        s = N.BatchStats()
        N.check(self._lib.tg_batch_stats_get(self._handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in N.BatchStats._fields_}
