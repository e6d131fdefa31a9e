"""numpy views of the reference's std430 parameter blocks (terraingen_b200/csrc/layouts.h).

The reference's host code builds these bytes for RunKernel; the dtypes here let Python build or
inspect them field by field (include/terraingen/noise/fractals.h:58, layers/kernels/craters.h:26-139).
"""

from __future__ import annotations

import numpy as np

# Fractal (fractals.h:58): a C++ bool, three padding bytes, then 12 four-byte fields.
FRACTAL = np.dtype([
    ("enabled", "u1"), ("pad", "u1", 3), ("seed", "<u4"), ("wavelength", "<f4"),
    ("amplitude", "<f4"), ("octaves", "<i4"), ("lacunarity", "<f4"), ("gain", "<f4"),
    ("basis", "<u4"), ("type", "<u4"), ("offset", "<f4"), ("blend", "<u4"),
    ("warpAmplitude", "<f4"), ("warpWavelength", "<f4"),
])
assert FRACTAL.itemsize == 52

NOISE_LAYER_KERNEL = np.dtype([("fractals", FRACTAL, 8), ("count", "<u4")])
assert NOISE_LAYER_KERNEL.itemsize == 420

_F, _U, _I = "<f4", "<u4", "<i4"

CRATER_PROFILE_KERNEL = np.dtype([
    ("simple", _U), ("rim", _U), ("complex", _U), ("diffused", _U), ("transitionDiameter", _F),
    ("floorCoefficient", _F), ("floorExponent", _F), ("peakHeightCoefficient", _F),
    ("peakHeightExponent", _F), ("peakWidthCoefficient", _F), ("peakWidthExponent", _F),
    ("peakFromVolume", _U), ("peakFitMaxDiameter", _F), ("ejectaExponent", _F),
    ("complexReachRadii", _F), ("tableExtent", _F), ("tableCells", _U), ("agesOffset", _U),
    ("ageCount", _U),
])
assert CRATER_PROFILE_KERNEL.itemsize == 76

CRATER_SHAPE_KERNEL = np.dtype([
    ("profile", CRATER_PROFILE_KERNEL), ("reachRadii", _F), ("profileReachRadii", _F),
    ("blendStart", _F), ("blendEnd", _F), ("blendShape", _U), ("interiorReplacement", _F),
    ("replaceStart", _F), ("replaceEnd", _F), ("mantling", _F), ("ejectaReachRadii", _F),
    ("rimSigma", _F), ("rimInner", _F), ("rimOuter", _F), ("rimStrength", _F), ("rimShape", _U),
    ("noiseAmplitude", _F), ("noiseWavelength", _F), ("noiseOctaves", _I), ("noiseGain", _F),
    ("noiseRimAmplitude", _F), ("noiseRimWavelength", _F), ("noiseRimInner", _F),
    ("noiseRimOuter", _F), ("wallStreaks", _F), ("wallStreakWidth", _F), ("ejecta", _F),
    ("ejectaLineation", _F), ("minFreshness", _F),
])
assert CRATER_SHAPE_KERNEL.itemsize == 188

CRATER_RECORD = np.dtype([
    ("x", _F), ("y", _F), ("diameter", _F), ("resolution", _F), ("freshDepth", _F),
    ("freshRim", _F), ("currentDepth", _F), ("currentRim", _F), ("diffusion", _F),
    ("ellipticity", _F), ("heading", _F), ("firstHarmonic", _U), ("harmonicCount", _U),
    ("harmonicOffset", _U), ("tableCount", _U), ("tableOffset", _U), ("profileOffset", _U),
    ("hasDatum", _U), ("datumA", _F), ("datumB", _F), ("datumC", _F), ("noiseKey", _U),
    ("textureKey", _U), ("markCount", _U), ("markOffset", _U), ("shiftX", _F), ("shiftY", _F),
    ("upslopeX", _F), ("upslopeY", _F), ("terraceCount", _U), ("terraceOffset", _U),
    ("peakCount", _U), ("peakOffset", _U), ("replace", _U), ("xLow", _F), ("yLow", _F),
])
assert CRATER_RECORD.itemsize == 144


def fractal(seed=0, wavelength=1000.0, amplitude=100.0, octaves=8, lacunarity=2.0, gain=0.5,
            basis=0, type=0, offset=1.0, blend=0, warp_amplitude=0.0, warp_wavelength=500.0,
            enabled=True) -> np.ndarray:
    """One `Fractal` with the reference's defaults (fractals.h:58-72)."""
    f = np.zeros((), FRACTAL)
    f["enabled"] = 1 if enabled else 0
    f["seed"] = seed
    f["wavelength"] = wavelength
    f["amplitude"] = amplitude
    f["octaves"] = octaves
    f["lacunarity"] = lacunarity
    f["gain"] = gain
    f["basis"] = basis
    f["type"] = type
    f["offset"] = offset
    f["blend"] = blend
    f["warpAmplitude"] = warp_amplitude
    f["warpWavelength"] = warp_wavelength
    return f


def noise_layer_kernel(fractals) -> np.ndarray:
    """`MakeNoiseLayerKernel` (noise_layer.h:45): the enabled fractals, in order, at most 8."""
    k = np.zeros((), NOISE_LAYER_KERNEL)
    n = 0
    for f in fractals:
        if f["enabled"] and n < 8:
            k["fractals"][n] = f
            n += 1
    k["count"] = n
    return k


def split(value: np.ndarray):
    """`SplitCoordinate` (crater_kernel.h): a double as a float and the float of its remainder."""
    value = np.asarray(value, np.float64)
    high = value.astype(np.float32)
    low = (value - high.astype(np.float64)).astype(np.float32)
    return high, low
