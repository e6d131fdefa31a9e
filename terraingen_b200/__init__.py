"""terraingen_b200: a B200 (sm_100a) CUDA backend for TerrainGen's per-cell terrain evaluation.

The product is libtgb200.so (C ABI in include/tgb200.h) with its hand-written kernels under csrc/
and the reference-side drop-in device under adapter/. This package builds it in-tree
(`python -m terraingen_b200.build`) and exposes it to Python through ctypes; it never falls back
to a CPU path.
"""

from .device import Device, GridSpec, centered, geographic_sphere_keys  # noqa: F401
from ._native import TgError, library  # noqa: F401
from . import layouts  # noqa: F401

__all__ = ["Device", "GridSpec", "centered", "TgError", "library", "layouts"]
