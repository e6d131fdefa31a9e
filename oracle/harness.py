"""ctypes access to the oracle: test infrastructure only.

The product never imports this module. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs use it, as the checker and the CPU baseline.

  - `restate()`  - oracle/_ref/libtgrestate.so, the FP32/FP64 restatement (oracle/restate.cpp);
  - `reference()` - oracle/_ref/libtgref.so, the reference CPU path built from its own sources;
  - `capture()`  - oracle/_ref/libtgref_capture.so, the reference pipeline recording what it hands
                   its GPU backend through the product's drop-in device;
  - `dropin()`   - oracle/_ref/libtgref_cuda.so, the reference pipeline on libtgb200 (GPU).
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"

_U32, _I32, _F, _D = C.c_uint32, C.c_int32, C.c_float, C.c_double


class Scene(C.Structure):
    """`tgref_scene` (oracle/ref_harness.cpp)."""

    _fields_ = [
        ("width", _U32), ("height", _U32), ("transform", _D * 6),
        ("source", _I32), ("elevation", _F), ("sourceFractals", _U32),
        ("sourceStack", C.c_ubyte * (52 * 8)),
        ("layerFractals", _U32), ("layerStack", C.c_ubyte * (52 * 8)),
        ("craters", _I32), ("seed", _U32),
        ("sfdCoefficient", _D), ("sfdExponent", _D), ("minDiameter", _D), ("maxDiameter", _D),
        ("lifetimeGyr", _D), ("depthRatio", _D), ("rimRatio", _D),
        ("profile", _I32), ("transitionDiameter", _D), ("applyPreset", _I32),
        ("noiseAmplitude", _D), ("rimNoiseAmplitude", _D), ("wallStreaks", _D), ("ejecta", _D),
        ("rimSigma", _D), ("terraceOnset", _D), ("terraceFull", _D),
        ("boulders", _I32), ("boulderSeed", _U32), ("boulderCoefficient", _D),
        ("boulderExponent", _D), ("boulderMin", _D), ("boulderMax", _D), ("heightRatio", _D),
        ("datum", _I32), ("interiorReplacement", _D), ("bodyRadius", _D),
        ("terraceMinFreshness", _D),
    ]


def make_scene(grid, source_fractals=None, elevation=0.0, layer_fractals=None, craters=None,
               boulders=None):
    """A Scene on `grid` (terraingen_b200.GridSpec). `craters` is a dict of crater-layer fields
    (seed, sfdCoefficient, sfdExponent, minDiameter, maxDiameter, lifetimeGyr, depthRatio,
    rimRatio, profile, transitionDiameter, applyPreset, noiseAmplitude, ...)."""
    s = Scene()
    s.width, s.height = grid.width, grid.height
    for i, v in enumerate(grid.transform()):
        s.transform[i] = v
    s.elevation = elevation
    if source_fractals is not None:
        fr = np.atleast_1d(source_fractals)
        s.source = 1
        s.sourceFractals = len(fr)
        C.memmove(s.sourceStack, fr.tobytes(), fr.nbytes)
    if layer_fractals is not None:
        fr = np.atleast_1d(layer_fractals)
        s.layerFractals = len(fr)
        C.memmove(s.layerStack, fr.tobytes(), fr.nbytes)
    if craters is not None:
        s.craters = 1
        defaults = dict(seed=1, sfdCoefficient=1e-3, sfdExponent=2.0, minDiameter=2.0,
                        maxDiameter=60.0, lifetimeGyr=1.0, depthRatio=0.2, rimRatio=0.04,
                        profile=0, transitionDiameter=15000.0, applyPreset=0,
                        noiseAmplitude=0.0, rimNoiseAmplitude=0.0, wallStreaks=0.0, ejecta=0.0,
                        rimSigma=0.0, terraceOnset=0.0, terraceFull=0.0, datum=0,
                        interiorReplacement=0.0, terraceMinFreshness=0.0)
        defaults.update(craters)
        for k, v in defaults.items():
            setattr(s, k, v)
    if boulders is not None:
        s.boulders = 1
        defaults = dict(boulderSeed=1, boulderCoefficient=0.05, boulderExponent=2.5,
                        boulderMin=0.2, boulderMax=3.0, heightRatio=0.5)
        defaults.update(boulders)
        for k, v in defaults.items():
            setattr(s, k, v)
    return s


def boulders(lib: C.CDLL, scene: Scene) -> np.ndarray:
    """The boulders the scene's boulder layer draws: [n, 5] (x, y, diameter, exposed, weight)."""
    n = lib.tgref_boulders(C.byref(scene), None, 0)
    if n < 0:
        raise RuntimeError(lib.tgref_error().decode())
    out = np.zeros((n, 5), np.float64)
    lib.tgref_boulders(C.byref(scene), out.ctypes.data, n)
    return out


def boulders_posed(lib: C.CDLL, scene: Scene, pose) -> np.ndarray:
    """tgref_boulders_posed: the layer's boulders with height ratio and burial drawn between
    bounds (min ratio, max ratio, min burial, max burial)."""
    pose = np.array(pose, np.float64)
    n = lib.tgref_boulders_posed(C.byref(scene), pose.ctypes.data, None, 0)
    if n < 0:
        raise RuntimeError(lib.tgref_error().decode())
    out = np.zeros((n, 5), np.float64)
    lib.tgref_boulders_posed(C.byref(scene), pose.ctypes.data, out.ctypes.data, n)
    return out


def below_boulders(lib: C.CDLL, scene: Scene, threads: int = 0) -> np.ndarray:
    out = np.zeros((scene.height, scene.width), np.float32)
    if lib.tgref_evaluate_below_boulders(C.byref(scene), threads, out.ctypes.data) != 0:
        raise RuntimeError(lib.tgref_error().decode())
    return out


def diamond_square(lib: C.CDLL, posts: np.ndarray, post_grid, grid, fractal_dimension: float,
                   scale: float, seed: int = 1, interp: int = 0, threads: int = 0,
                   backend: int = 0):
    """(heights [h, w] float32, ms): the reference's DiamondSquareUpsampler through a RasterSource,
    evaluated on Backend::Cpu (0) or Backend::Cuda (1)."""
    posts = np.ascontiguousarray(posts, np.float32)
    ph, pw = posts.shape
    pt = np.array(post_grid.transform(), np.float64)
    ot = np.array(grid.transform(), np.float64)
    out = np.zeros((grid.height, grid.width), np.float32)
    ms = _D()
    if lib.tgref_ds_on(backend, posts.ctypes.data, pw, ph, pt.ctypes.data, fractal_dimension,
                       scale, interp, seed, grid.width, grid.height, ot.ctypes.data, threads,
                       out.ctypes.data, C.byref(ms)) != 0:
        raise RuntimeError(lib.tgref_error().decode())
    return out, ms.value


def seam(lib: C.CDLL, earlier: np.ndarray, later: np.ndarray, transform, mode: int,
         width: float = 50.0, decay: float = 50.0) -> dict:
    """The reference's seam between two rasters on one grid (tgref_seam): the lattice's size and
    transform, the samples the solve starts from (data, difference) and the field's posts."""
    earlier = np.ascontiguousarray(earlier, np.float32)
    later = np.ascontiguousarray(later, np.float32)
    h, w = earlier.shape
    t = np.array(transform, np.float64)
    pad = 64 + int(np.ceil(max(width, 3.0 * decay) / min(abs(t[1]), abs(t[5])))) + 3
    capacity = (w + 2 * pad) * (h + 2 * pad)
    data = np.zeros(capacity, np.uint8)
    diff = np.zeros(capacity, np.float32)
    field = np.zeros(capacity, np.float32)
    lw, lh, lt, ms = C.c_uint32(), C.c_uint32(), np.zeros(6), C.c_double()
    st = lib.tgref_seam(earlier.ctypes.data, later.ctypes.data, w, h, t.ctypes.data, mode,
                        width, decay, C.addressof(lw), C.addressof(lh), lt.ctypes.data,
                        data.ctypes.data, diff.ctypes.data, field.ctypes.data, capacity,
                        C.addressof(ms))
    if st != 0:
        raise RuntimeError(f"tgref_seam failed ({st}): {lib.tgref_error().decode()}")
    n = lw.value * lh.value
    shape = (lh.value, lw.value)
    return {"width": lw.value, "height": lh.value, "transform": lt,
            "data": data[:n].reshape(shape), "difference": diff[:n].reshape(shape),
            "field": field[:n].reshape(shape), "ms": ms.value}


def body_noise(lib: C.CDLL, fractals, elevation: float, radius: float, grid) -> np.ndarray:
    """The reference's SyntheticSource heights on a sphere (tgref_body_noise) for `grid`
    (terraingen_b200.GridSpec in degrees)."""
    fr = np.ascontiguousarray(np.atleast_1d(fractals))
    t = np.ascontiguousarray(grid.transform(), np.float64)
    out = np.zeros((grid.height, grid.width), np.float32)
    if lib.tgref_body_noise(fr.ctypes.data, len(fr), elevation, radius, grid.width, grid.height,
                            t.ctypes.data, out.ctypes.data) != 0:
        raise RuntimeError(lib.tgref_error().decode())
    return out


def write_crater_list(lib: C.CDLL, path, x, y, diameter, age, ids, manual, replace,
                      json: bool) -> None:
    """The reference's WriteCraterList (tgref_write_crater_list) without attributes."""
    cols = [np.ascontiguousarray(v, np.float64) for v in (x, y, diameter, age)]
    i = np.ascontiguousarray(ids, np.uint64)
    m = np.ascontiguousarray(manual, np.uint8)
    r = np.ascontiguousarray(replace, np.uint8)
    st = lib.tgref_write_crater_list(str(path).encode(), *[c.ctypes.data for c in cols],
                                     i.ctypes.data, m.ctypes.data, r.ctypes.data, len(i),
                                     int(json))
    if st != 0:
        raise RuntimeError(f"tgref_write_crater_list failed: {lib.tgref_error().decode()}")


BOULDER_DOUBLES = ("x", "y", "diameter", "height", "burial", "yaw", "lean", "tilt",
                   "tilt_azimuth", "wear", "ground")


def write_boulder_list(lib: C.CDLL, path, columns: dict, json: bool) -> None:
    """The reference's WriteBoulderList (tgref_write_boulder_list). `columns` holds the doubles
    named in BOULDER_DOUBLES (angles in radians; NaN grounds are unset) and id, parent, piece,
    rest and model."""
    values = np.ascontiguousarray(np.stack([np.asarray(columns[k], np.float64)
                                            for k in BOULDER_DOUBLES]))
    n = values.shape[1]
    known = np.ascontiguousarray(np.isfinite(values[10]), np.uint8)
    ids = np.ascontiguousarray(columns["id"], np.uint64)
    parent = np.ascontiguousarray(columns["parent"], np.uint64)
    piece = np.ascontiguousarray(columns["piece"], np.uint32)
    rest = np.ascontiguousarray(columns["rest"], np.uint8)
    model = np.ascontiguousarray(columns["model"], np.uint8)
    st = lib.tgref_write_boulder_list(str(path).encode(), values.ctypes.data, known.ctypes.data,
                                      ids.ctypes.data, parent.ctypes.data, piece.ctypes.data,
                                      rest.ctypes.data, model.ctypes.data, n, int(json))
    if st != 0:
        raise RuntimeError(f"tgref_write_boulder_list failed: {lib.tgref_error().decode()}")


COMPRESSION = {"none": 0, "lzw": 1, "packbits": 2, "deflate": 3}  # TiffCompression's order


def write_geotiff(lib: C.CDLL, path, bands: list, transform, nodata=None, directory=(),
                  doubles=(), ascii: str = "", compression: str = "lzw", tile_size: int = 256,
                  big_tiff: bool = False) -> None:
    """The reference's WriteGeoTiff (tgref_write_geotiff) of float bands sharing one grid;
    `nodata` None, NaN or a value."""
    arrays = [np.ascontiguousarray(b, np.float32) for b in bands]
    h, w = arrays[0].shape
    ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    t = np.ascontiguousarray(transform, np.float64)
    mode = 0 if nodata is None else (1 if np.isnan(nodata) else 2)
    d = np.ascontiguousarray(directory, np.uint16)
    dp = np.ascontiguousarray(doubles, np.float64)
    st = lib.tgref_write_geotiff(str(path).encode(), C.cast(ptrs, C.c_void_p), len(arrays), w, h,
                                 t.ctypes.data, mode, 0.0 if mode != 2 else float(nodata),
                                 d.ctypes.data, len(d), dp.ctypes.data, len(dp), ascii.encode(),
                                 COMPRESSION[compression], tile_size, int(big_tiff))
    if st != 0:
        raise RuntimeError(f"tgref_write_geotiff failed: {lib.tgref_error().decode()}")


def chain(lib: C.CDLL, earlier: np.ndarray, later: np.ndarray, transform, mode: int,
          width: float, decay: float, out_grid) -> np.ndarray:
    """A SourceChain of the two rasters joined by `mode`, evaluated on `out_grid`."""
    earlier = np.ascontiguousarray(earlier, np.float32)
    later = np.ascontiguousarray(later, np.float32)
    h, w = earlier.shape
    t = np.array(transform, np.float64)
    ot = np.array(out_grid.transform(), np.float64)
    out = np.zeros((out_grid.height, out_grid.width), np.float32)
    st = lib.tgref_chain(earlier.ctypes.data, later.ctypes.data, w, h, t.ctypes.data, mode,
                         width, decay, out_grid.width, out_grid.height, ot.ctypes.data,
                         out.ctypes.data)
    if st != 0:
        raise RuntimeError(f"tgref_chain failed: {lib.tgref_error().decode()}")
    return out


def patch_chain(lib: C.CDLL, rasters: list, grids: list, mode: int, width: float, decay: float,
                out_grid) -> np.ndarray:
    """A SourceChain of raster patches, each on its own grid (tgref_patch_chain), on `out_grid`."""
    rasters = [np.ascontiguousarray(r, np.float32) for r in rasters]
    n = len(rasters)
    ptrs = (C.c_void_p * n)(*[r.ctypes.data for r in rasters])
    widths = np.array([g.width for g in grids], np.uint32)
    heights = np.array([g.height for g in grids], np.uint32)
    transforms = np.array([g.transform() for g in grids], np.float64).ravel()
    ot = np.array(out_grid.transform(), np.float64)
    out = np.zeros((out_grid.height, out_grid.width), np.float32)
    st = lib.tgref_patch_chain(n, C.cast(ptrs, C.c_void_p), widths.ctypes.data,
                               heights.ctypes.data, transforms.ctypes.data, mode, width, decay,
                               out_grid.width, out_grid.height, ot.ctypes.data, out.ctypes.data)
    if st != 0:
        raise RuntimeError(f"tgref_patch_chain failed: {lib.tgref_error().decode()}")
    return out


def config1_craters() -> dict:
    """The 257 x 257, 1 m crater scene (2000 craters expected over the extent, N(>D) ~ D^-2 on
    [2, 60] m, depth/diameter 0.2, rim 0.04 D, uniform ages over 1 Gyr, seed 1)."""
    area = 257.0 * 257.0
    c = 2000.0 / (area * (2.0 ** -2.0 - 60.0 ** -2.0))
    return dict(seed=1, sfdCoefficient=c, sfdExponent=2.0, minDiameter=2.0, maxDiameter=60.0,
                lifetimeGyr=1.0, depthRatio=0.2, rimRatio=0.04, profile=0, applyPreset=0)


def build(target: str = "all") -> None:
    """Builds oracle/_ref (needs the reference sources; the restatement needs none)."""
    subprocess.run(["make", "-C", str(HERE), "-j8", target], check=True,
                   stdout=subprocess.DEVNULL)


_libs: dict = {}


def _load(name: str) -> C.CDLL:
    if name not in _libs:
        path = REF / name
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (make -C oracle)")
        _libs[name] = C.CDLL(str(path))
    return _libs[name]


def available(name: str) -> bool:
    return (REF / name).exists()


def restate() -> C.CDLL:
    lib = _load("libtgrestate.so")
    lib.rs_pcg.restype = _U32
    lib.rs_pcg.argtypes = [_U32]
    lib.rs_pcg3d.argtypes = [_U32, _U32, _U32, C.c_void_p]
    lib.rs_perlin2_f32.restype = _F
    lib.rs_perlin2_f32.argtypes = [_F, _F, _U32]
    lib.rs_perlin2_f64.restype = _D
    lib.rs_perlin2_f64.argtypes = [_D, _D, _U32]
    lib.rs_fbm2_f32.restype = _F
    lib.rs_fbm2_f32.argtypes = [_F, _F, _U32, _F, _F, C.c_int, _F, _F]
    lib.rs_fbm2_f64.restype = _D
    lib.rs_fbm2_f64.argtypes = [_D, _D, _U32, _D, _D, C.c_int, _D, _D]
    lib.rs_fbm_grid_f32.argtypes = [_U32, _U32, _D, _D, _D, _U32, _F, _F, C.c_int, _F, _F, _F,
                                    C.c_void_p]
    lib.rs_fbm_grid_f64.argtypes = [_U32, _U32, _D, _D, _D, _U32, _D, _D, C.c_int, _D, _D, _D,
                                    C.c_void_p]
    lib.rs_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rs_ds_normal.restype = _D
    lib.rs_ds_normal.argtypes = [C.c_int64, C.c_int64, C.c_int, _U32]
    lib.rs_crater_profile_f64.restype = _D
    lib.rs_crater_profile_f64.argtypes = [C.c_int, _U32, _D, _D, _D, _D, _D, _D]
    return lib


def _harness(name: str) -> C.CDLL:
    lib = _load(name)
    lib.tgref_evaluate.argtypes = [C.POINTER(Scene), C.c_int, C.c_uint, C.c_void_p,
                                   C.POINTER(_D)]
    lib.tgref_evaluate.restype = C.c_int
    lib.tgref_error.restype = C.c_char_p
    lib.tgref_craters.argtypes = [C.POINTER(Scene), C.c_void_p, _D, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]
    lib.tgref_craters.restype = C.c_long
    if hasattr(lib, "tgref_points"):
        lib.tgref_points.argtypes = [C.POINTER(Scene), C.c_void_p, _U32, _D, C.c_void_p]
        lib.tgref_points.restype = C.c_int
    lib.tgref_boulders.argtypes = [C.POINTER(Scene), C.c_void_p, C.c_long]
    lib.tgref_boulders.restype = C.c_long
    if hasattr(lib, "tgref_datum_relief"):
        lib.tgref_datum_relief.argtypes = [C.c_void_p] * 8 + [_U32, _U32, _U32, C.c_void_p]
        lib.tgref_datum_relief.restype = C.c_int
    if hasattr(lib, "tgref_boulders_posed"):
        lib.tgref_boulders_posed.argtypes = [C.POINTER(Scene), C.c_void_p, C.c_void_p, C.c_long]
        lib.tgref_boulders_posed.restype = C.c_long
    lib.tgref_evaluate_below_boulders.argtypes = [C.POINTER(Scene), C.c_uint, C.c_void_p]
    lib.tgref_evaluate_below_boulders.restype = C.c_int
    lib.tgref_ds.argtypes = [C.c_void_p, _U32, _U32, C.c_void_p, _D, _D, C.c_int, _U32, _U32, _U32,
                             C.c_void_p, C.c_uint, C.c_void_p, C.POINTER(_D)]
    lib.tgref_ds.restype = C.c_int
    lib.tgref_ds_on.argtypes = [C.c_int] + lib.tgref_ds.argtypes
    lib.tgref_ds_on.restype = C.c_int
    lib.tgref_hook_calls.restype = C.c_long
    if hasattr(lib, "tgref_seam"):
        P = C.c_void_p
        lib.tgref_seam.argtypes = [P, P, _U32, _U32, P, C.c_int, _D, _D, P, P, P, P, P, P,
                                   C.c_size_t, P]
        lib.tgref_seam.restype = C.c_int
        lib.tgref_chain.argtypes = [P, P, _U32, _U32, P, C.c_int, _D, _D, _U32, _U32, P, P]
        lib.tgref_chain.restype = C.c_int
        lib.tgref_patch_chain.argtypes = [_U32, P, P, P, P, C.c_int, _D, _D, _U32, _U32, P, P]
        lib.tgref_patch_chain.restype = C.c_int
    if hasattr(lib, "tgref_write_geotiff"):
        P = C.c_void_p
        lib.tgref_write_geotiff.argtypes = [C.c_char_p, P, _U32, _U32, _U32, P, C.c_int, C.c_float,
                                            P, _U32, P, _U32, C.c_char_p, C.c_int, _U32, C.c_int]
        lib.tgref_write_geotiff.restype = C.c_int
    if hasattr(lib, "tgref_body_noise"):
        lib.tgref_body_noise.argtypes = [C.c_void_p, _U32, C.c_float, _D, _U32, _U32, C.c_void_p,
                                         C.c_void_p]
        lib.tgref_body_noise.restype = C.c_int
    if hasattr(lib, "tgref_write_crater_list"):
        P = C.c_void_p
        lib.tgref_write_crater_list.argtypes = [C.c_char_p, P, P, P, P, P, P, P, C.c_size_t,
                                                C.c_int]
        lib.tgref_write_crater_list.restype = C.c_int
    if hasattr(lib, "tgref_write_boulder_list"):
        P = C.c_void_p
        lib.tgref_write_boulder_list.argtypes = [C.c_char_p, P, P, P, P, P, P, P, C.c_size_t,
                                                 C.c_int]
        lib.tgref_write_boulder_list.restype = C.c_int
    return lib


def reference() -> C.CDLL:
    return _harness("libtgref.so")


def dropin() -> C.CDLL:
    return _harness("libtgref_cuda.so")


def hook_calls(lib: C.CDLL) -> int:
    """How many CPU-only pipeline stages the drop-in build has run on the device so far."""
    return int(lib.tgref_hook_calls())


def capture() -> C.CDLL:
    lib = _harness("libtgref_capture.so")
    lib.tgref_capture_count.restype = C.c_int
    lib.tgref_capture_info.argtypes = [C.c_int, C.c_void_p]
    lib.tgref_capture_field.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_size_t)]
    return lib


def evaluate(lib: C.CDLL, scene: Scene, backend: int = 0, threads: int = 0):
    """(heights [height, width] float32, milliseconds) from the harness `lib`."""
    out = np.zeros((scene.height, scene.width), np.float32)
    ms = _D()
    if lib.tgref_evaluate(C.byref(scene), backend, threads, out.ctypes.data, C.byref(ms)) != 0:
        raise RuntimeError(lib.tgref_error().decode())
    return out, ms.value


def points(lib: C.CDLL, scene: Scene, xy: np.ndarray, spacing: float) -> np.ndarray:
    """The scene's heights (float32) at the (x, y) rows of `xy` through the reference's point path
    (Terrain::HeightsAt -> EvaluatePoints) at sample `spacing`."""
    xy = np.ascontiguousarray(xy, np.float64).reshape(-1, 2)
    out = np.zeros(len(xy), np.float32)
    if lib.tgref_points(C.byref(scene), xy.ctypes.data, len(xy), spacing, out.ctypes.data) != 0:
        raise RuntimeError(lib.tgref_error().decode())
    return out


def craters(lib: C.CDLL, scene: Scene, region, spacing: float = 0.0) -> dict:
    """The crater population the scene's layer generates over region (x0, y0, x1, y1)."""
    reg = np.asarray(region, np.float64)
    n = lib.tgref_craters(C.byref(scene), reg.ctypes.data, spacing, None, None, None, None, None,
                          0)
    if n < 0:
        raise RuntimeError(lib.tgref_error().decode())
    out = {k: np.zeros(n, np.float64) for k in ("x", "y", "diameter", "age")}
    out["id"] = np.zeros(n, np.uint64)
    lib.tgref_craters(C.byref(scene), reg.ctypes.data, spacing, out["x"].ctypes.data,
                      out["y"].ctypes.data, out["diameter"].ctypes.data, out["age"].ctypes.data,
                      out["id"].ctypes.data, n)
    return out


CRATER_FIELDS = ["kernel", "records", "data", "heads", "entries", "xs", "x_lows", "ys", "y_lows",
                 "heights"]
NOISE_FIELDS = ["kernel", "xs", "ys", "heights"]


DATUM_FIELDS = ["kernel", "records", "data", "band_floats", "band_cells", "cells", "entries",
                "targets", "heights"]


def datum_relief(lib: C.CDLL, call: dict) -> np.ndarray:
    """The reference's KernelDatumRelief over a captured tg_crater_datums call (tgref_datum_relief):
    the lattice strip's heights after the relief is added."""
    heights = call["heights"].view(np.float32).copy()
    f = {k: np.ascontiguousarray(call[k]) for k in DATUM_FIELDS[:8]}
    st = lib.tgref_datum_relief(f["kernel"].ctypes.data, f["records"].ctypes.data,
                                f["data"].ctypes.data, f["band_floats"].ctypes.data,
                                f["band_cells"].ctypes.data, f["cells"].ctypes.data,
                                f["entries"].ctypes.data, f["targets"].ctypes.data, call["width"],
                                call["rows"], call["first_row"], heights.ctypes.data)
    if st != 0:
        raise RuntimeError(lib.tgref_error().decode())
    return heights


def captured(lib: C.CDLL) -> list:
    """Every captured backend call as a dict of numpy arrays."""
    calls = []
    for call in range(lib.tgref_capture_count()):
        info = np.zeros(8, np.uint32)
        lib.tgref_capture_info(call, info.ctypes.data)
        kind = int(info[0])
        names = {2: CRATER_FIELDS, 3: DATUM_FIELDS}.get(kind, NOISE_FIELDS)
        rec = {"kind": kind, "width": int(info[1]), "rows": int(info[2]),
               "first_row": int(info[3]), "nodata_mode": int(info[4]),
               "nodata_value": float(info[5:6].view(np.float32)[0])}
        for f, name in enumerate(names):
            ptr, size = C.c_void_p(), C.c_size_t()
            lib.tgref_capture_field(call, f, C.byref(ptr), C.byref(size))
            buf = (C.c_ubyte * size.value).from_address(ptr.value) if size.value else b""
            rec[name] = np.frombuffer(bytes(buf), np.uint8).copy()
        calls.append(rec)
    lib.tgref_capture_clear()
    return calls
