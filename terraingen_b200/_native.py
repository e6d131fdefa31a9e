"""ctypes bindings of libtgb200.so (include/tgb200.h).

Loading fails loudly: there is no CPU fallback, so a missing or unloadable library is an error
the caller sees, never a silent change of code path.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "lib" / "libtgb200.so"

TG_MEMORY_HOST = 0
TG_MEMORY_DEVICE = 1

STATUS = {0: "ok", 1: "argument", 2: "cuda", 3: "unsupported", 4: "memory", 5: "timeout",
          6: "state"}


class TgError(RuntimeError):
    """A tg_* call failed; `status` is its tg_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Grid(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("origin_x", C.c_double),
                ("pixel_width", C.c_double), ("row_rotation", C.c_double),
                ("origin_y", C.c_double), ("col_rotation", C.c_double),
                ("pixel_height", C.c_double)]


class NoData(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("value", C.c_float)]


_P = C.c_void_p
_U32 = C.c_uint32
_SZ = C.c_size_t
_I = C.c_int
_D = C.c_double
_F = C.c_float

# name -> argument types; every function returns int except where noted.
SIGNATURES = {
    "tg_open": [_I, C.POINTER(_P)],
    "tg_close": [_P],
    "tg_last_error": [],
    "tg_device_name": [_P, C.c_char_p, _SZ],
    "tg_synchronize": [_P],
    "tg_set_wait_limit": [_P, _U32],
    "tg_set_host_threads": [C.c_uint],
    "tg_noise_layer": [_P, _P, _SZ, C.POINTER(Grid), _D, _D, _P, NoData, _I, _P],
    "tg_noise_layer_rows": [_P, _P, _SZ, _P, _P, _U32, _U32, _P, NoData, _I, _P],
    "tg_noise_source": [_P, _P, _U32, _F, C.POINTER(Grid), _P, _I, _P],
    "tg_noise_probe": [_P, _P, _U32, _U32, _P, _P, _I],
    "tg_noise_source_body": [_P, _P, _U32, _F, C.POINTER(Grid), _D, _P, _I, _P],
    "tg_craters_apply": [_P, _P, _SZ, _P, _U32, _P, _U32, _P, C.POINTER(Grid), _P, NoData, _I,
                         _P],
    "tg_craters_apply_lists": [_P, _P, _SZ, _P, _U32, _P, _U32, _P, _U32, _P, _U32, _P, _P, _P,
                               _P, _U32, _U32, _U32, _P, NoData, _I, _P],
    "tg_craters_apply_body": [_P, _P, _SZ, _P, _U32, _P, _U32, _P, _P, _U32, _P, _U32, _P, _U32,
                              _U32, _U32, _P, NoData, _I, _P],
}

class Population(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("sfd_coefficient", C.c_double),
                ("sfd_exponent", C.c_double), ("min_diameter", C.c_double),
                ("max_diameter", C.c_double), ("lifetime_gyr", C.c_double),
                ("depth_ratio", C.c_double), ("rim_ratio", C.c_double),
                ("cutoff_depth_ratio", C.c_double), ("cell_size_factor", C.c_double),
                ("margin_radii", C.c_double), ("min_resolved_diameter", C.c_double)]


class Shaping(C.Structure):
    _fields_ = [("profile", C.c_uint32), ("irregular", C.c_uint32),
                ("transition_diameter", C.c_double), ("terrace_onset", C.c_double),
                ("terrace_full", C.c_double), ("terrace_min_freshness", C.c_double)]


class BoulderPopulation(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("sfd_coefficient", C.c_double),
                ("sfd_exponent", C.c_double), ("min_diameter", C.c_double),
                ("max_diameter", C.c_double), ("min_height_ratio", C.c_double),
                ("max_height_ratio", C.c_double), ("min_burial", C.c_double),
                ("max_burial", C.c_double), ("fade_start_samples", C.c_double),
                ("fade_end_samples", C.c_double), ("cell_size_factor", C.c_double)]


class DsOptions(C.Structure):
    _fields_ = [("fractal_dimension", _D), ("scale", _D), ("interp", _U32), ("seed", _U32),
                ("min_pixel_size", _D)]


class Terrain(C.Structure):
    _fields_ = [("fractals", _P), ("n_fractals", _U32), ("elevation", _F), ("noise_layer", _P),
                ("crater_kernel", _P), ("crater_records", _P), ("n_craters", _U32),
                ("crater_data", _P), ("n_crater_data", _U32), ("crater_footprints", _P),
                ("boulders", _P), ("n_boulders", _U32), ("boulder_width", _D)]


SIGNATURES.update({
    "tg_evaluate": [_P, C.POINTER(Terrain), C.POINTER(Grid), _P, _I, _P],
    "tg_measure_alu": [_P, C.POINTER(_D)],
    "tg_device_counters": [_P, _P, _SZ],
    "tg_ds_refine": [_P, _P, _U32, _U32, C.POINTER(Grid), C.POINTER(DsOptions), C.POINTER(Grid),
                     _P, _I, _P],
    "tg_ds_refine_window": [_P, _P, C.c_int64, C.c_int64, _U32, _U32, C.POINTER(Grid),
                            C.POINTER(DsOptions), C.POINTER(Grid), _P, _I, _P],
    "tg_philox_probe": [_P, _P, _U32, _P, _P],
    "tg_boulders_bake": [_P, _P, _U32, _D, C.POINTER(Grid), _P, NoData, _I, _P],
    "tg_boulders_bake_static": [_P, _U32, _D, C.POINTER(Grid), _P, NoData, _P, C.c_char_p, _SZ],
    "tg_crater_generate": [C.POINTER(Population), _P, _P, _P, _P, _P, _P, _SZ,
                             C.POINTER(_SZ)],
    "tg_boulder_generate": [C.POINTER(BoulderPopulation), _P, _D, _P, _SZ, C.POINTER(_SZ)],
    "tg_crater_generate_device": [_P, C.POINTER(Population), _P, _P, _P, _P, _P, _P, _SZ,
                                  C.POINTER(_SZ), _D, _I, _P],
    "tg_crater_batch": [C.POINTER(Population), C.POINTER(Shaping), C.POINTER(Grid), _P, _P, _SZ,
                        _P, _SZ, _P, C.POINTER(_SZ), C.POINTER(_SZ)],
    "tg_crater_batch_device": [_P, C.POINTER(Population), C.POINTER(Shaping), C.POINTER(Grid),
                               _P, _P, _SZ, _P, _SZ, _P, C.POINTER(_SZ), C.POINTER(_SZ),
                               C.POINTER(_SZ), _P],
})

class Tile(C.Structure):
    _fields_ = [("grid", Grid), ("height_offset", C.c_uint64), ("pitch", _U32),
                ("crater_begin", _U32), ("crater_count", _U32), ("data_begin", _U32),
                ("boulder_begin", _U32), ("boulder_count", _U32), ("boulder_width", _D)]


class PointSet(C.Structure):
    _fields_ = [("point_begin", _U32), ("point_count", _U32), ("height_offset", C.c_uint64),
                ("crater_begin", _U32), ("crater_count", _U32), ("data_begin", _U32),
                ("boulder_begin", _U32), ("boulder_count", _U32), ("reserved", _U32),
                ("boulder_width", _D)]


class BatchInput(C.Structure):
    _fields_ = [("tiles", _P), ("n_tiles", _U32), ("fractals", _P), ("n_fractals", _U32),
                ("elevation", _F), ("crater_kernel", _P), ("crater_records", _P),
                ("n_craters", _U32), ("crater_data", _P), ("n_crater_data", _U32),
                ("crater_footprints", _P), ("boulders", _P), ("n_boulders", _U32),
                ("point_sets", _P), ("n_point_sets", _U32), ("points", _P), ("n_points", _U32)]


class BatchStats(C.Structure):
    _fields_ = [("variant", _U32), ("bin_width", _U32), ("bin_height", _U32),
                ("cells_per_thread", _U32), ("fast", _U32), ("bins", _U32),
                ("cells", C.c_uint64), ("crater_pairs", C.c_uint64),
                ("boulder_pairs", C.c_uint64), ("crater_entries", C.c_uint64),
                ("boulder_entries", C.c_uint64), ("captures", _U32), ("replays", _U32),
                ("bin_ms", _F), ("evaluate_ms", _F), ("graph_ms", _F), ("ctas", _U32)]


SIGNATURES.update({
    "tg_batch_create": [_P, C.POINTER(_P)],
    "tg_batch_destroy": [_P],
    "tg_batch_load": [_P, C.POINTER(BatchInput)],
    "tg_batch_evaluate": [_P, _P, _SZ, _I, _P],
    "tg_batch_run": [_P, C.POINTER(BatchInput), _P, _SZ, _I, _P],
    "tg_batch_tune": [_P, _I, _P],
    "tg_batch_variant_count": [],
    "tg_batch_set_variant": [_P, _I],
    "tg_batch_variant": [_I, C.POINTER(_U32), C.POINTER(_U32), C.POINTER(_U32)],
    "tg_batch_stats_get": [_P, C.POINTER(BatchStats)],
})

class SeamOptions(C.Structure):
    _fields_ = [("mode", _U32), ("levels", _U32), ("sweeps", _U32), ("coarsest_sweeps", _U32),
                ("width", _D), ("decay_length", _D), ("tolerance", _D)]


class SeamStats(C.Structure):
    _fields_ = [("unknowns", _U32), ("levels", _U32), ("iterations", _U32), ("reserved", _U32),
                ("prepare_ms", _D), ("solve_ms", _D)]


SIGNATURES.update({
    "tg_seam_solve": [_P, _P, _P, _U32, _U32, _D, _D, C.POINTER(SeamOptions), _P, _I, _P],
    "tg_seam_stats_get": [C.POINTER(SeamStats)],
    "tg_crater_datums": [_P, _P, _SZ, _P, _U32, _P, _U32, _P, _U32, _P, _U32, _P, _U32, _P, _U32,
                         _P, _U32, _U32, _U32, _U32, _P, _I, _P],
    "tg_crater_body_datums": [_P, _P, _SZ, _P, _U32, _P, _U32, _P, _P, _P, _U32, _P, _U32, _P,
                              _U32, _U32, _U32, _P, NoData, _I, _P],
    "tg_seam_fill": [_P, _P, C.POINTER(Grid), _P, C.POINTER(Grid), _P, NoData, _P, _I, _P],
    "tg_seam_samples": [_P, _P, _P, C.POINTER(Grid), C.c_int64, C.c_int64, _U32, _U32, NoData,
                        _P, _P, _I, _P],
})


class ServerOptions(C.Structure):
    _fields_ = [("fractals", _P), ("n_fractals", _U32), ("elevation", _F),
                ("craters", Population), ("shaping", Shaping), ("base_spacing", _D),
                ("point_spacing", _D), ("hbm_budget", C.c_uint64),
                ("max_batch_cells", C.c_uint64), ("slots", _U32), ("region_cells", _U32),
                ("variant", C.c_int32), ("reserved", _U32), ("post_spacing", _D),
                ("refine", DsOptions)]


class Request(C.Structure):
    _fields_ = [("id", C.c_uint64), ("kind", _U32), ("memory", _U32), ("grid", Grid),
                ("points", _P), ("n_points", _U32), ("heights", _P)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("cells", C.c_uint64), ("regions_built", C.c_uint64),
                ("regions_evicted", C.c_uint64), ("regions_resident", C.c_uint64),
                ("feature_bytes", C.c_uint64), ("device_bytes", C.c_uint64),
                ("peak_bytes", C.c_uint64), ("deferred", C.c_uint64), ("gpu_ms", _D),
                ("region_ms", _D)]


SIGNATURES.update({
    "tg_server_create": [_P, C.POINTER(ServerOptions), C.POINTER(_P)],
    "tg_server_destroy": [_P],
    "tg_server_submit": [_P, C.POINTER(Request)],
    "tg_server_poll": [_P, _I, _P, _SZ, C.POINTER(_SZ)],
    "tg_server_stats_get": [_P, C.POINTER(ServerStats)],
})

class GeotiffOptions(C.Structure):
    """tg_geotiff_options (GeoTiffWriteOptions)."""

    _fields_ = [("compression", C.c_uint32), ("tile_size", C.c_uint32), ("big_tiff", C.c_uint32),
                ("reserved", C.c_uint32)]


class GeoKeys(C.Structure):
    """tg_geokeys (GeoKeys: the three GeoTIFF key tags' values)."""

    _fields_ = [("directory", _P), ("directory_count", C.c_uint32), ("double_count", C.c_uint32),
                ("double_params", _P), ("ascii_params", C.c_char_p)]


SIGNATURES.update({
    "tg_geotiff_write": [_P, C.c_char_p, _P, C.c_uint32, C.POINTER(Grid), NoData,
                         C.POINTER(GeoKeys), C.POINTER(GeotiffOptions), _I, _P],
})

RESTYPES = {"tg_close": None, "tg_last_error": C.c_char_p, "tg_batch_destroy": None,
            "tg_set_host_threads": None,
            "tg_server_destroy": None}

_lib = None


def library() -> C.CDLL:
    """The loaded libtgb200.so, with argument types set; raises if it cannot be loaded."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(
                f"{LIBRARY} is missing: build it with `python -m terraingen_b200.build` "
                "(there is no CPU fallback)")
        lib = C.CDLL(str(LIBRARY))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = RESTYPES.get(name, C.c_int)
        _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    """The C ABI names the header declares (every one must be exported)."""
    return list(SIGNATURES)


def check(status: int) -> None:
    if status != 0:
        raise TgError(status, library().tg_last_error().decode())
