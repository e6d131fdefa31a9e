// Device-side crater shaping: the height one crater adds at a cell, from its std430 record and
// the shared float data, restating the shaping functions of TerrainGen's crater kernel header
// (include/terraingen/layers/kernels/craters.h:152-1370). Each function names the reference
// function it follows; the formulas, constants and branch order are kept, since the heights must
// agree with the reference's CPU path to 1e-3 m.
//
// Differences by design: records and data are read through the read-only cache, and the
// transcendental functions are CUDA's own (cosf, atan2f, expf, powf, logf), which agree with the
// host libm to a few ulp.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "layouts.h"
#include "noise_math.cuh"

namespace tgb {
namespace crater {

using noise::sclamp;
using noise::smax;
using noise::smin;

__device__ __forceinline__ float value(const float* __restrict__ data, uint32_t i) {
    return __ldg(data + i);
}

// a - b for coordinates held as a float and the float of its remainder (craters.h:152).
__device__ __forceinline__ float split_difference(float a, float aLow, float b, float bLow) {
    return (a - b) + (aLow - bLow);
}

// asin(s) / s (craters.h:160).
__device__ __forceinline__ float arcsine_ratio(float s) {
    if (s < 0.25f) {
        const float s2 = s * s;
        return 1.0f + s2 * (1.0f / 6.0f +
                            s2 * (3.0f / 40.0f + s2 * (5.0f / 112.0f + s2 * (35.0f / 1152.0f))));
    }
    return atan2f(s, sqrtf(1.0f - s * s)) / s;
}

struct Offset {
    float dx, dy;
};

// `KernelFrameOffset` (craters.h:170).
__device__ __forceinline__ Offset frame_offset(const CraterFrame& f, float dx, float dy,
                                               float dz) {
    Offset o;
    o.dx = dx * f.eastX + dy * f.eastY + dz * f.eastZ;
    o.dy = dx * f.northX + dy * f.northY + dz * f.northZ;
    if (f.sphereRadius > 0.0f) {
        const float chord = sqrtf(dx * dx + dy * dy + dz * dz);
        const float arc = chord * arcsine_ratio(smin(0.5f * chord / f.sphereRadius, 1.0f));
        const float across = sqrtf(o.dx * o.dx + o.dy * o.dy);
        if (across > 0.0f) {
            o.dx *= arc / across;
            o.dy *= arc / across;
        } else {
            o.dy = arc;
        }
    }
    return o;
}

// `KernelFalloffShape` (craters.h:248).
__device__ __forceinline__ float falloff_shape(float t, uint32_t shape) {
    if (shape == 0u) {
        return 1.0f - t;
    }
    if (shape == 1u) {
        return 1.0f - t * t * (3.0f - 2.0f * t);
    }
    if (shape == 2u) {
        return 1.0f - t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f);
    }
    const float tail = expf(-4.5f);
    const float z = 3.0f * t;
    return (expf(-0.5f * z * z) - tail) / (1.0f - tail);
}

// `KernelFalloff` (craters.h:264).
__device__ __forceinline__ float falloff(float x, float start, float end, uint32_t shape) {
    if (x <= start) {
        return 1.0f;
    }
    if (x >= end) {
        return 0.0f;
    }
    return falloff_shape((x - start) / (end - start), shape);
}

__device__ __forceinline__ float smoothstep(float t) {  // craters.h:275
    const float u = sclamp(t, 0.0f, 1.0f);
    return u * u * (3.0f - 2.0f * u);
}

// Direction from east, 0 at the origin (craters.h:282).
__device__ __forceinline__ float angle(float dy, float dx) {
    if (dx == 0.0f && dy == 0.0f) {
        return 0.0f;
    }
    return atan2f(dy, dx);
}

#define TGB_PI 3.14159265358979f
#define TGB_TWO_PI 6.28318530717959f

struct PeriodicCell {
    uint32_t index;
    float t;
};

// `KernelPeriodicAt` (craters.h:300).
__device__ __forceinline__ PeriodicCell periodic_at(float turns, uint32_t size) {
    const float position = (turns - floorf(turns)) * float(size);
    PeriodicCell c;
    c.index = min(uint32_t(position), size - 1u);
    c.t = position - float(c.index);
    return c;
}

__device__ __forceinline__ float ejecta_scale(float radius) {  // craters.h:309
    return 0.14f * powf(radius, 0.74f);
}

__device__ __forceinline__ float ejecta_share(float radii, float reachRadii) {  // craters.h:315
    if (radii <= 1.0f) {
        return 1.0f;
    }
    if (radii >= reachRadii) {
        return 0.0f;
    }
    const float atReach = 1.0f / (reachRadii * reachRadii * reachRadii);
    return (1.0f / (radii * radii * radii) - atReach) / (1.0f - atReach);
}

// `FassettThomsonExterior` (craters.h:330).
__device__ __forceinline__ float ft_exterior(float x, float start) {
    const float polynomial =
        0.188253307f + x * (-0.187050452f + x * (0.01844746f + x * 0.01505647f));
    const float u = (x - start) / (1.5f - start);
    return polynomial * (1.0f - u * u);
}

// `FassettThomsonShape` (craters.h:338).
__device__ __forceinline__ float ft_shape(float x, uint32_t rim, float freshRim,
                                          float currentDepth) {
    if (x > 1.5f) {
        return 0.0f;
    }
    const float interior =
        -0.228809953f + x * (0.227533882f + x * (0.083116795f - x * 0.039499407f));
    float h = 0.0f;
    if (rim == 2u) {
        if (x <= 0.98f) {
            h = interior;
        } else if (x <= 1.02f) {
            h = freshRim;
        } else {
            h = ft_exterior(x, 1.02f);
        }
    } else {
        const float edge = rim == 0u ? 0.98f : 1.0f;
        if (x <= 0.2f) {
            h = -0.181f;
        } else if (x <= edge) {
            h = interior;
        } else {
            h = ft_exterior(x, edge);
        }
    }
    return smax(h, freshRim - currentDepth);
}

struct ProfilePoint {
    float height, slope;
};

// `MartinParkesDunstanExterior` (craters.h:375).
__device__ __forceinline__ ProfilePoint mpd_exterior(float x, float rim, float ejectaScale) {
    const float offset = rim - ejectaScale;
    const float gradient = -ejectaScale / 8.0f - offset;
    const float r = 1.0f / (x + 1.0f);
    const float law = ejectaScale * r * r * r + offset + gradient * x;
    const float lawSlope = -3.0f * ejectaScale * r * r * r * r + gradient;
    const float taper = 1.0f - x * x;
    return ProfilePoint{law * taper, lawSlope * taper - 2.0f * x * law};
}

// `MartinParkesDunstanHeight` (craters.h:389), on the depth and rim ratios given.
__device__ __forceinline__ float mpd_height(float distance, float diameter, float freshRimRatio,
                                            float depthRatio, float rimRatio) {
    const float depth = depthRatio * diameter;
    const float rim = rimRatio * diameter;
    const float freshRim = freshRimRatio * diameter;
    const float radius = 0.5f * diameter;
    const float x = distance / radius - 1.0f;
    if (x >= 1.0f) {
        return 0.0f;
    }
    const float k = freshRim - rim + depth;
    const float alpha = (rim - freshRim) / k;
    if (x <= alpha) {
        return (k * x + 2.0f * k) * x + freshRim;
    }
    if (x <= 0.0f) {
        return k * (alpha + 1.0f) / alpha * x * x + rim;
    }
    const float es =
        freshRim > 0.0f ? ejecta_scale(radius) * rim / freshRim : ejecta_scale(radius);
    const float beta = smin(1.0f, 1.5f * (freshRim - rim) / k);
    if (x <= beta) {
        const ProfilePoint join = mpd_exterior(beta, rim, es);
        const float drop = rim - join.height;
        const float slope = drop > 0.0f ? smax(join.slope, -3.0f * drop / beta) : join.slope;
        const float t = x / beta;
        return rim + (join.height - rim) * t * t * (3.0f - 2.0f * t) +
               beta * slope * t * t * (t - 1.0f);
    }
    return mpd_exterior(x, rim, es).height;
}

// The depth and rim ratios a profile reads: the current state, or the fresh one where the
// reference evaluates a copy of the record with the fresh ratios (craters.h:507-512).
struct State {
    float freshDepth, freshRim, currentDepth, currentRim;
};

__device__ __forceinline__ float simple_height(const CraterProfileKernel& p, float distance,
                                               float diameter, const State& s) {  // :425
    if (p.simple == kProfileMartinParkesDunstan) {
        return mpd_height(distance, diameter, s.freshRim, s.currentDepth, s.currentRim);
    }
    return ft_shape(distance / (0.5f * diameter), p.rim, s.freshRim, s.currentDepth) * diameter;
}

__device__ __forceinline__ float kilometer_law(float coefficient, float exponent, float diameter,
                                               bool volume) {  // craters.h:435
    const float kilometers = coefficient * powf(diameter / 1000.0f, exponent);
    return volume ? kilometers * 1e9f : kilometers * 1000.0f;
}

struct PeakSize {
    float height, base;
};

__device__ __forceinline__ PeakSize complex_peak(const CraterProfileKernel& p,
                                                 float diameter) {  // craters.h:448
    const float fitted =
        p.peakFitMaxDiameter > 0.0f ? smin(diameter, p.peakFitMaxDiameter) : diameter;
    PeakSize size;
    size.height = kilometer_law(p.peakHeightCoefficient, p.peakHeightExponent, fitted, false);
    if (p.peakFromVolume == 1u) {
        const float volume = kilometer_law(p.peakWidthCoefficient, p.peakWidthExponent, fitted, true);
        size.base = sqrtf(3.0f * volume / (TGB_PI * size.height));
    } else {
        size.base = 0.5f * kilometer_law(p.peakWidthCoefficient, p.peakWidthExponent, fitted, false);
    }
    size.base *= diameter / fitted;
    return size;
}

__device__ __forceinline__ float peak_dome(PeakSize size, float distance) {  // craters.h:465
    if (!(distance < size.base)) {
        return 0.0f;
    }
    const float u = 1.0f - (distance / size.base) * (distance / size.base);
    return size.height * u * u;
}

__device__ __forceinline__ float kept_depth(const State& s) {  // craters.h:474
    return s.freshDepth > 0.0f ? s.currentDepth / s.freshDepth : 1.0f;
}

__device__ __forceinline__ float complex_height(const CraterProfileKernel& p, float distance,
                                                float diameter, const State& s) {  // :479
    const float radius = 0.5f * diameter;
    const float x = distance / radius;
    const float depth = s.currentDepth * diameter;
    const float rim = s.currentRim * diameter;
    if (x >= 1.0f) {
        if (x >= p.complexReachRadii) {
            return 0.0f;
        }
        const float edge = powf(p.complexReachRadii, -p.ejectaExponent);
        return rim * (powf(x, -p.ejectaExponent) - edge) / (1.0f - edge);
    }
    const float floorShare =
        smin(0.9f, kilometer_law(p.floorCoefficient, p.floorExponent, diameter, false) / diameter);
    float height = rim - depth;
    if (x > floorShare) {
        const float t = (x - floorShare) / (1.0f - floorShare);
        height += depth * t * t;
    }
    return height + kept_depth(s) * peak_dome(complex_peak(p, diameter), distance);
}

__device__ __forceinline__ float fresh_height(const CraterProfileKernel& p, float distance,
                                              float diameter, const State& s) {  // :501
    if (p.complex == 1u && diameter >= p.transitionDiameter) {
        return complex_height(p, distance, diameter, s);
    }
    return simple_height(p, distance, diameter, s);
}

struct TableCell {
    uint32_t index;
    float t;
};

__device__ __forceinline__ TableCell table_at(const CraterProfileKernel& p, float x) {  // :516
    const float position = x / p.tableExtent * float(p.tableCells);
    TableCell c;
    c.index = min(uint32_t(position), p.tableCells - 1u);
    c.t = position - float(c.index);
    return c;
}

__device__ __forceinline__ float table_lerp(const float* data, uint32_t at, float t) {  // :525
    return (1.0f - t) * value(data, at) + t * value(data, at + 1u);
}

struct AgeRow {
    uint32_t row;
    float weight;
};

// `KernelAgeRowAt` (craters.h:538).
__device__ __forceinline__ AgeRow age_row_at(const CraterProfileKernel& p, const float* data,
                                             float tau) {
    AgeRow age{0u, 0.0f};
    const uint32_t last = p.ageCount - 1u;
    const float first = value(data, p.agesOffset + 1u);
    if (tau >= value(data, p.agesOffset + last)) {
        age.row = last;
    } else if (tau < first) {
        age.weight = tau / first;
    } else {
        uint32_t low = 1u, high = last;
        while (high - low > 1u) {
            const uint32_t middle = (low + high) / 2u;
            if (value(data, p.agesOffset + middle) <= tau) {
                low = middle;
            } else {
                high = middle;
            }
        }
        age.row = low;
        const float below = value(data, p.agesOffset + low);
        const float above = value(data, p.agesOffset + high);
        age.weight = logf(tau / below) / logf(above / below);
    }
    return age;
}

// `DiffusedProfileHeight` (craters.h:584).
__device__ __forceinline__ float diffused_height(const CraterProfileKernel& p, const float* data,
                                                 float distance, float diameter,
                                                 const CraterRecord& c, const State& s) {
    if (!(c.diffusion > 0.0f)) {
        const State fresh{s.freshDepth, s.freshRim, s.freshDepth, s.freshRim};
        return fresh_height(p, distance, diameter, fresh);
    }
    const float x = distance / diameter;
    if (x >= p.tableExtent) {
        return 0.0f;
    }
    const TableCell cell = table_at(p, x);
    const AgeRow age = age_row_at(p, data, c.diffusion);
    const uint32_t width = p.tableCells + 1u;
    const uint32_t at = c.profileOffset + age.row * width + cell.index;
    float v = table_lerp(data, at, cell.t);
    if (age.weight > 0.0f) {
        v += age.weight * (table_lerp(data, at + width, cell.t) - v);
    }
    return diameter * v;
}

// `TabulatedProfileHeight` (craters.h:601).
__device__ __forceinline__ float tabulated_height(const CraterProfileKernel& p, const float* data,
                                                  float distance, float diameter,
                                                  const CraterRecord& c) {
    const float x = distance / diameter;
    if (!(x < p.tableExtent)) {
        return 0.0f;
    }
    const TableCell cell = table_at(p, x);
    return diameter * table_lerp(data, c.profileOffset + cell.index, cell.t);
}

// `KernelProfileHeight` (craters.h:612).
__device__ __forceinline__ float profile_height(const CraterShapeKernel& k, const float* data,
                                                float distance, float diameter,
                                                const CraterRecord& c, const State& s) {
    if (k.profile.simple == kProfileTabulated) {
        return tabulated_height(k.profile, data, distance, diameter, c);
    }
    if (k.profile.diffused == 1u) {
        return diffused_height(k.profile, data, distance, diameter, c, s);
    }
    return fresh_height(k.profile, distance, diameter, s);
}

// `KernelRoundedHeight` (craters.h:628): the profile with its rim rounded by a Gaussian.
static __device__ __noinline__ float rounded_height(const CraterShapeKernel& k, const float* data,
                                             float distance, float diameter, const CraterRecord& c,
                                             const State& s) {
    const float height = profile_height(k, data, distance, diameter, c, s);
    if (k.rimSigma == 0.0f) {
        return height;
    }
    const float radius = 0.5f * diameter;
    const float radii = distance / radius;
    const float weight =
        radii <= 1.0f ? k.rimStrength * falloff(2.0f - radii, 1.0f, 2.0f - k.rimInner, k.rimShape)
                      : k.rimStrength * falloff(radii, 1.0f, k.rimOuter, k.rimShape);
    if (weight == 0.0f) {
        return height;
    }
    const float sigma = k.rimSigma * radius;
    const float step = 0.5f * sigma;
    const float position = (distance - radius) / step;
    const float first = floorf(position) - 7.0f;
    float smoothed = 0.0f, total = 0.0f;
    for (int i = 0; i < 16; ++i) {
        const float node = first + float(i);
        const float z = 0.5f * (node - position);
        const float w = expf(-0.5f * z * z) * falloff(fabsf(z), 3.0f, 4.0f, 2u);
        smoothed += w * profile_height(k, data, fabsf(radius + step * node), diameter, c, s);
        total += w;
    }
    return height + weight * (smoothed / total - height);
}

// Perlin fBm with the fields `KernelFractalParams` (craters.h:658) fixes.
__device__ __forceinline__ FractalParams kernel_fractal(uint32_t seed, float wavelength,
                                                        int octaves, float gain) {
    return FractalParams{seed, wavelength, 1.0f, octaves, 2.0f, gain, kBasisPerlin, kTypeFbm, 1.0f};
}

// `KernelNoiseHeight` (craters.h:673).
static __device__ __noinline__ float noise_height(const CraterShapeKernel& k, const CraterRecord& c,
                                           float dx, float dy, float radii) {
    if (k.noiseAmplitude == 0.0f && k.noiseRimAmplitude == 0.0f) {
        return 0.0f;
    }
    const float radius = 0.5f * c.diameter;
    const float footprint = radii <= 1.0f ? 1.0f : falloff(radii, 1.0f, k.profileReachRadii, 2u);
    const float rim = radii <= 1.0f ? falloff(2.0f - radii, 1.0f, 2.0f - k.noiseRimInner, 2u)
                                    : falloff(radii, 1.0f, k.noiseRimOuter, 2u);
    float height = 0.0f;
    if (k.noiseAmplitude > 0.0f && footprint > 0.0f) {
        const FractalParams p =
            kernel_fractal(c.noiseKey, k.noiseWavelength * radius, k.noiseOctaves, k.noiseGain);
        height += k.noiseAmplitude * footprint * noise::fractal2(dx, dy, p);
    }
    if (k.noiseRimAmplitude > 0.0f && rim > 0.0f) {
        const FractalParams p = kernel_fractal(c.noiseKey + 1u, k.noiseRimWavelength * radius,
                                               k.noiseOctaves, k.noiseGain);
        height += k.noiseRimAmplitude * rim * noise::fractal2(dx, dy, p);
    }
    return c.diameter * height;
}

// `KernelRadialStreaks` (craters.h:698).
__device__ __forceinline__ float radial_streaks(float radii, float theta, float across,
                                                float along, int octaves, uint32_t seed) {
    const float ring = 1.0f / across;
    return noise::perlin_fbm3_float(ring * cosf(theta), ring * sinf(theta), radii / along, seed,
                                    octaves, 0.5f);
}

// `KernelTextureHeight` (craters.h:706).
static __device__ __noinline__ float texture_height(const CraterShapeKernel& k, const CraterRecord& c,
                                             float dx, float dy, float radii) {
    if (k.wallStreaks == 0.0f && k.ejecta == 0.0f) {
        return 0.0f;
    }
    const float freshness = c.freshDepth > 0.0f ? c.currentDepth / c.freshDepth : 1.0f;
    const float fade = smoothstep((freshness - k.minFreshness) / (1.0f - k.minFreshness));
    if (!(fade > 0.0f)) {
        return 0.0f;
    }
    const float theta = angle(dy, dx);
    float height = 0.0f;
    if (k.wallStreaks > 0.0f && radii > 0.25f && radii < 1.0f) {
        const float band =
            smoothstep((radii - 0.25f) / 0.35f) * smoothstep((1.0f - radii) / 0.1f);
        height += k.wallStreaks * c.diameter * band *
                  radial_streaks(radii, theta, k.wallStreakWidth, 0.5f, 2, c.textureKey);
    }
    if (k.ejecta > 0.0f && radii > 1.0f && radii < k.ejectaReachRadii) {
        const float radius = 0.5f * c.diameter;
        const float thickness = ejecta_scale(radius) * ejecta_share(radii, k.ejectaReachRadii);
        const float rise = smoothstep((radii - 1.0f) / 0.1f);
        height += k.ejecta * thickness * rise *
                  radial_streaks(radii, theta, k.ejectaLineation, 2.0f * k.ejectaLineation, 3,
                                 c.textureKey + 1u);
    }
    return fade * height;
}

// `KernelEllipseScale` (craters.h:737).
__device__ __forceinline__ float ellipse_scale(float theta, float ellipticity, float heading) {
    const float along = sqrtf(ellipticity);
    const float across = 1.0f / along;
    const float u = cosf(theta - heading) / along;
    const float v = sinf(theta - heading) / across;
    return 1.0f / sqrtf(u * u + v * v);
}

__device__ __forceinline__ float catmull_rom(float p0, float p1, float p2, float p3,
                                             float t) {  // craters.h:746
    return 0.5f * (2.0f * p1 + (p2 - p0) * t + (2.0f * p0 - 5.0f * p1 + 4.0f * p2 - p3) * t * t +
                   (3.0f * (p1 - p2) + p3 - p0) * t * t * t);
}

__device__ __forceinline__ float marks_window(float radii, float inner, float outer,
                                              float fade) {  // craters.h:753
    if (!(radii > inner - fade) || !(radii < outer + fade)) {
        return 0.0f;
    }
    return smoothstep((radii - inner + fade) / fade) * smoothstep((outer + fade - radii) / fade);
}

#define TGB_TABLE_FINE_FADE 6.5f  // craters.h:763 kTableFineFade

// `KernelOutlineScaleAt` (craters.h:771).
__device__ __forceinline__ float outline_scale_at(const float* data, const CraterRecord& c,
                                                  float dx, float dy, float share) {
    const float theta = angle(dy, dx);
    const float scale =
        c.ellipticity != 1.0f ? ellipse_scale(theta, c.ellipticity, c.heading) : 1.0f;
    float wobble = 1.0f;
    if (c.tableCount > 0u && share > 0.0f) {
        const PeriodicCell cell = periodic_at(theta / TGB_TWO_PI, c.tableCount);
        const float rim = (1.0f - cell.t) * value(data, c.tableOffset + cell.index) +
                          cell.t * value(data, c.tableOffset + (cell.index + 1u) % c.tableCount);
        if (share >= 1.0f) {
            wobble += share * rim;
        } else {
            float broad = 0.0f;
            for (uint32_t n = 0u; n < c.harmonicCount; ++n) {
                const float order = float(c.firstHarmonic + n);
                const float wave = value(data, c.harmonicOffset + 2u * n) *
                                   cosf(order * theta + value(data, c.harmonicOffset + 2u * n + 1u));
                broad += wave;
                wobble += powf(share, 0.5f * order) * wave;
            }
            wobble += powf(share, TGB_TABLE_FINE_FADE) * (rim - broad);
        }
    } else if (share > 0.0f) {
        for (uint32_t n = 0u; n < c.harmonicCount; ++n) {
            const float order = float(c.firstHarmonic + n);
            const float kept = share < 1.0f ? powf(share, 0.5f * order) : 1.0f;
            wobble += kept * value(data, c.harmonicOffset + 2u * n) *
                      cosf(order * theta + value(data, c.harmonicOffset + 2u * n + 1u));
        }
    }
    return scale * wobble;
}

__device__ __forceinline__ float outline_share(float radii) {  // craters.h:818
    return smoothstep(radii);
}

__device__ __forceinline__ float worn_outline_share(const CraterRecord& c) {  // craters.h:825
    return c.freshRim > 0.0f ? sclamp(c.currentRim / c.freshRim, 0.0f, 1.0f) : 1.0f;
}

// `KernelMarkShift` (craters.h:831).
__device__ __forceinline__ float mark_shift(const float* data, const CraterRecord& c, float dx,
                                            float dy, float radii) {
    const float window = marks_window(radii, value(data, c.markOffset),
                                      value(data, c.markOffset + 1u), value(data, c.markOffset + 2u));
    if (window == 0.0f) {
        return 0.0f;
    }
    const uint32_t size = c.markCount;
    const PeriodicCell cell = periodic_at(angle(dy, dx) / TGB_TWO_PI, size);
    const uint32_t index = cell.index;
    const uint32_t knots = c.markOffset + 3u;
    return window * catmull_rom(value(data, knots + (index + size - 1u) % size),
                                value(data, knots + index),
                                value(data, knots + (index + 1u) % size),
                                value(data, knots + (index + 2u) % size), cell.t);
}

// --- terraces (craters.h:851-1024) -----------------------------------------------------------

#define TGB_TERRACE_HEADER 20u
#define TGB_TERRACE_SCARP 8u
#define TGB_TERRACE_STEP 3u
#define TGB_TERRACE_BLOCK_BLEND 0.3f

__device__ __forceinline__ float terrace_block_value(uint32_t key, int cell, int count,
                                                     float gaps) {  // craters.h:879
    const int wrapped = ((cell % count) + count) % count;
    const float hash = noise::unit(noise::pcg(key + uint32_t(wrapped) * 0x9E3779B9u));
    return gaps < 0.0f ? hash : (hash >= gaps ? 1.0f : 0.0f);
}

__device__ __forceinline__ float terrace_blocks(const float* data, uint32_t s, float theta,
                                                uint32_t salt, float gaps) {  // craters.h:887
    const float turns = value(data, s + 2u) * theta / TGB_TWO_PI + value(data, s + 3u);
    const int count = int(value(data, s + 2u));
    const uint32_t key = uint32_t(value(data, s + 7u)) ^ (salt * 0x85EBCA6Bu);
    const float cellStart = floorf(turns);
    const int cell = int(cellStart);
    const float u = turns - cellStart;
    const float v = terrace_block_value(key, cell, count, gaps);
    if (u < TGB_TERRACE_BLOCK_BLEND) {
        const float b = smoothstep(0.5f + 0.5f * u / TGB_TERRACE_BLOCK_BLEND);
        return terrace_block_value(key, cell - 1, count, gaps) * (1.0f - b) + v * b;
    }
    if (u > 1.0f - TGB_TERRACE_BLOCK_BLEND) {
        const float b = smoothstep(0.5f + 0.5f * (1.0f - u) / TGB_TERRACE_BLOCK_BLEND);
        return terrace_block_value(key, cell + 1, count, gaps) * (1.0f - b) + v * b;
    }
    return v;
}

__device__ __forceinline__ float harmonics(const float* data, uint32_t offset, uint32_t first,
                                           uint32_t count, float theta, float turn) {  // :910
    float sum = 0.0f;
    for (uint32_t n = 0u; n < count; ++n) {
        const float order = float(first + n);
        sum += value(data, offset + 2u * n) *
               cosf(order * (theta + turn) + value(data, offset + 2u * n + 1u));
    }
    return sum;
}

__device__ __forceinline__ float terrace_arc(const float* data, uint32_t o, float theta,
                                             float step) {  // craters.h:924
    const float cut = value(data, o + 4u);
    if (!(cut > -1.5f)) {
        return 1.0f;
    }
    const float arcs = harmonics(data, o + 6u, 2u, 5u, theta, 2.39996323f * step);
    return smoothstep((arcs - cut) / value(data, o + 5u));
}

__device__ __forceinline__ float terrace_base(const float* data, const CraterRecord& c,
                                              uint32_t k) {  // craters.h:935
    if (k == 0u) {
        return 0.0f;
    }
    if (k >= c.terraceCount) {
        return 1.0f;
    }
    return value(data, c.terraceOffset + TGB_TERRACE_HEADER + TGB_TERRACE_SCARP * (k - 1u));
}

__device__ __forceinline__ float terrace_scarp(const float* data, const CraterRecord& c,
                                               uint32_t k, float theta) {  // craters.h:951
    if (k == 0u || k >= c.terraceCount) {
        return terrace_base(data, c, k);
    }
    const uint32_t s = c.terraceOffset + TGB_TERRACE_HEADER + TGB_TERRACE_SCARP * (k - 1u);
    const float turns = value(data, s + 2u) * theta / TGB_TWO_PI + value(data, s + 3u);
    const float f = 2.0f * (turns - floorf(turns)) - 1.0f;
    const float scallop = value(data, s + 1u) * (1.0f - f * f - 2.0f / 3.0f);
    const float wobble = value(data, s + 4u) * cosf(3.0f * theta + value(data, s + 5u));
    const float block = 2.0f * terrace_blocks(data, s, theta, 0u, -1.0f) - 1.0f;
    return value(data, s) + scallop + wobble + value(data, s + 6u) * block;
}

__device__ __forceinline__ float terrace_rim_scale(const float* data, const CraterRecord& c,
                                                   float theta) {  // craters.h:968
    const uint32_t o = c.terraceOffset;
    const float turns = value(data, o + 17u) * theta / TGB_TWO_PI + value(data, o + 18u);
    const float f = 2.0f * (turns - floorf(turns)) - 1.0f;
    return 1.0f + value(data, o + 16u) * (1.0f - f * f - 2.0f / 3.0f);
}

__device__ __forceinline__ float terrace_ease(float v, float rounding) {  // craters.h:979
    const float steepest = 1.0f / (1.0f - 0.5f * rounding);
    if (v < rounding) {
        return steepest * v * v / (2.0f * rounding);
    }
    return steepest * (v - 0.5f * rounding);
}

// `KernelTerracedRadii` (craters.h:990).
static __device__ __noinline__ float terraced_radii(const float* data, const CraterRecord& c, float radii,
                                             float theta) {
    const uint32_t o = c.terraceOffset;
    const float inner = value(data, o);
    if (!(radii > inner) || !(radii < 1.0f)) {
        return radii;
    }
    const float t = (radii - inner) / (1.0f - inner);
    uint32_t step = 0u;
    float low = 0.0f;
    float high = terrace_scarp(data, c, 1u, theta);
    while (step + 1u < c.terraceCount && t >= high) {
        ++step;
        low = high;
        high = terrace_scarp(data, c, step + 1u, theta);
    }
    const float within = sclamp((t - low) / (high - low), 0.0f, 1.0f);
    float strength = value(data, o + 2u) * terrace_arc(data, o, theta, float(step));
    if (c.terraceCount > 1u) {
        const bool top = step + 1u >= c.terraceCount;
        const uint32_t k = top ? step : step + 1u;
        const uint32_t s = o + TGB_TERRACE_HEADER + TGB_TERRACE_SCARP * (k - 1u);
        strength *= terrace_blocks(data, s, theta, top ? 2u : 1u, value(data, o + 19u));
    }
    const float rounding = value(data, o + 3u);
    const float slope = value(data, o + 1u);
    const uint32_t s = o + TGB_TERRACE_HEADER + TGB_TERRACE_SCARP * (c.terraceCount - 1u) +
                       TGB_TERRACE_STEP * step;
    const float level = value(data, s);
    const float scarp = value(data, s + 1u);
    strength *= value(data, s + 2u);
    const float lower = scarp * level;
    const float upper = scarp * (1.0f - level);
    float stair = level;
    if (within < lower) {
        stair = level * (1.0f - terrace_ease(1.0f - within / lower, rounding));
    } else if (within > 1.0f - upper) {
        stair = level + (1.0f - level) * terrace_ease((within - (1.0f - upper)) / upper, rounding);
    }
    const float rise = slope * within + (1.0f - slope) * stair;
    const float shaped = within + strength * (rise - within);
    const float from = terrace_base(data, c, step);
    const float to = terrace_base(data, c, step + 1u);
    return inner + (from + shaped * (to - from)) * (1.0f - inner);
}

// `KernelProfileDistance` (craters.h:1028).
__device__ __forceinline__ float profile_distance(const float* data, const CraterRecord& c,
                                                  float dx, float dy) {
    float distance = sqrtf(dx * dx + dy * dy);
    if (c.ellipticity != 1.0f || c.harmonicCount > 0u || c.tableCount > 0u || c.markCount > 0u) {
        const float share = outline_share(distance / (0.5f * c.diameter)) * worn_outline_share(c);
        distance /= outline_scale_at(data, c, dx, dy, share);
    }
    if (c.markCount > 0u) {
        const float radius = 0.5f * c.diameter;
        distance += radius * mark_shift(data, c, dx, dy, distance / radius);
    }
    if (c.terraceCount > 0u) {
        const float radius = 0.5f * c.diameter;
        const float theta = angle(dy, dx);
        const float scale = terrace_rim_scale(data, c, theta);
        distance /= 1.0f + (scale - 1.0f) * outline_share(distance / radius);
        distance = radius * terraced_radii(data, c, distance / radius, theta);
    }
    return distance;
}

__device__ __forceinline__ float slope_shift_weight(const CraterRecord& c, float dx,
                                                    float dy) {  // craters.h:1051
    const float radii = sqrtf(dx * dx + dy * dy) / (0.5f * c.diameter);
    return 1.0f - smoothstep((radii - 0.3f) / 0.7f);
}

__device__ __forceinline__ float slope_raised_share(const CraterRecord& c, float dx,
                                                    float dy) {  // craters.h:1058
    const float distance = sqrtf(dx * dx + dy * dy);
    if (!(distance > 0.0f)) {
        return 1.0f;
    }
    const float removed = sqrtf(c.upslopeX * c.upslopeX + c.upslopeY * c.upslopeY);
    const float cosine = smax(0.0f, (c.upslopeX * dx + c.upslopeY * dy) / (removed * distance));
    return 1.0f - removed * cosine * cosine;
}

__device__ __forceinline__ float shifted_distance(const float* data, const CraterRecord& c,
                                                  float dx, float dy) {  // craters.h:1070
    const float shift =
        c.shiftX != 0.0f || c.shiftY != 0.0f ? slope_shift_weight(c, dx, dy) : 0.0f;
    return profile_distance(data, c, dx - shift * c.shiftX, dy - shift * c.shiftY);
}

__device__ __forceinline__ float upslope_height(const CraterRecord& c, float height, float dx,
                                                float dy) {  // craters.h:1077
    if (height > 0.0f && (c.upslopeX != 0.0f || c.upslopeY != 0.0f)) {
        return height * slope_raised_share(c, dx, dy);
    }
    return height;
}

// --- central peak massifs (craters.h:1086-1183) ----------------------------------------------

#define TGB_PEAK_HEADER 6u
#define TGB_PEAK_MASSIF 11u
#define TGB_PEAK_REACH 2.6f

__device__ __forceinline__ float peak_massif(const float* data, uint32_t m, float px,
                                             float py) {  // craters.h:1104
    const float ex = px - value(data, m);
    const float ey = py - value(data, m + 1u);
    const float radius = value(data, m + 2u);
    const float stretch = value(data, m + 3u);
    const float cosine = value(data, m + 4u);
    const float sine = value(data, m + 5u);
    const float qx = (ex * cosine + ey * sine) / (radius * stretch);
    const float qy = (ey * cosine - ex * sine) * stretch / radius;
    const float squared = qx * qx + qy * qy;
    if (!(squared < 1.0f)) {
        return 0.0f;
    }
    const float pull = 1.0f - squared;
    const float sx = qx - value(data, m + 8u) * pull;
    const float sy = qy - value(data, m + 9u) * pull;
    const float r = smin(sqrtf(sx * sx + sy * sy), 1.0f);
    const float flank = 1.0f - powf(r, value(data, m + 7u));
    return value(data, m + 6u) * powf(flank, value(data, m + 10u));
}

static __device__ __noinline__ float peak_massifs(const float* data, const CraterRecord& c, PeakSize size,
                                           float dx, float dy) {  // craters.h:1128
    const uint32_t o = c.peakOffset;
    float px = dx / size.base;
    float py = dy / size.base;
    const float roughness = value(data, o);
    const float wavelength = value(data, o + 1u);
    const float warp = value(data, o + 2u);
    const uint32_t key = uint32_t(value(data, o + 3u));
    if (warp > 0.0f) {
        const FractalParams shape = kernel_fractal(key + 1u, 2.0f * wavelength, 3, 0.5f);
        const float wx = noise::fractal2(px, py, shape);
        const float wy = noise::fractal2(px + 17.31f, py - 9.73f, shape);
        px += warp * wx;
        py += warp * wy;
    }
    float height = 0.0f;
    for (uint32_t n = 0u; n < c.peakCount; ++n) {
        height = smax(height, peak_massif(data, o + TGB_PEAK_HEADER + TGB_PEAK_MASSIF * n, px, py));
    }
    if (roughness > 0.0f && height > 0.0f) {
        FractalParams ridges = kernel_fractal(key, wavelength, 5, 0.5f);
        ridges.type = kTypeRidged;
        height *= 1.0f + roughness * noise::fractal2(px, py, ridges);
    }
    return size.height * height;
}

// `KernelPeakRelief` (craters.h:1161).
__device__ __forceinline__ float peak_relief(const CraterShapeKernel& k, const float* data,
                                             const CraterRecord& c, const State& s,
                                             float distance, float dx, float dy) {
    if (c.peakCount == 0u || k.profile.complex != 1u || k.profile.diffused == 1u ||
        k.profile.simple == kProfileTabulated || c.diameter < k.profile.transitionDiameter) {
        return 0.0f;
    }
    const PeakSize size = complex_peak(k.profile, c.diameter);
    PeakSize scaled = size;
    scaled.height *= value(data, c.peakOffset + 4u);
    scaled.base *= value(data, c.peakOffset + 5u);
    const float shift =
        c.shiftX != 0.0f || c.shiftY != 0.0f ? slope_shift_weight(c, dx, dy) : 0.0f;
    const float sx = dx - shift * c.shiftX;
    const float sy = dy - shift * c.shiftY;
    const float reach = TGB_PEAK_REACH * smax(size.base, scaled.base);
    if (!(sx * sx + sy * sy < reach * reach)) {
        return 0.0f;
    }
    return kept_depth(s) * (peak_massifs(data, c, scaled, sx, sy) - peak_dome(size, distance));
}

// What crater `c` adds at (dx, dy) from its center, without the running height: the reference's
// `ApplyCraterKernel` (craters.h:1186) returns height + resolution * (shaped + replaced); without
// a datum the added part does not depend on the height, which is what lets the caller sum it
// compensated and in any order. `reached` is false beyond the crater's reach.
struct Contribution {
    float shaped;        // resolution * shaped relief
    float replaceWeight; // resolution * weight of the datum blend; 0 without a datum
    bool reached;
};

__device__ __forceinline__ Contribution crater_contribution(const CraterShapeKernel& k,
                                                            const float* data,
                                                            const CraterRecord& c, float dx,
                                                            float dy) {
    Contribution out{0.0f, 0.0f, false};
    const float diameter = c.diameter;
    const float radius = 0.5f * diameter;
    const float distance = shifted_distance(data, c, dx, dy);
    if (distance >= k.reachRadii * radius) {
        return out;
    }
    out.reached = true;
    const State s{c.freshDepth, c.freshRim, c.currentDepth, c.currentRim};
    const float radii = distance / radius;
    if (c.hasDatum == 1u) {
        float weight = c.replace == 1u
                           ? falloff(radii, k.replaceStart, k.replaceEnd, k.blendShape)
                           : k.interiorReplacement *
                                 falloff(radii, k.blendStart, k.blendEnd, k.blendShape);
        if (k.mantling > 0.0f && radii > 1.0f) {
            weight = smax(weight, k.mantling * ejecta_share(radii, k.ejectaReachRadii));
        }
        out.replaceWeight = weight;
    }
    const float bare =
        upslope_height(c, rounded_height(k, data, distance, diameter, c, s), dx, dy) +
        peak_relief(k, data, c, s, distance, dx, dy);
    const float shaped =
        bare + noise_height(k, c, dx, dy, radii) + texture_height(k, c, dx, dy, radii);
    out.shaped = c.resolution * shaped;
    return out;
}

// The reference's sequential form (craters.h:1186), for craters with a datum, whose blend reads
// the running height.
__device__ __forceinline__ float apply_with_datum(const CraterRecord& c, const Contribution& q,
                                                  float height, float dx, float dy) {
    const float replaced = q.replaceWeight * (c.datumA + c.datumB * dx + c.datumC * dy - height);
    return height + q.shaped + c.resolution * replaced;
}

// --- the common case, evaluated lean ----------------------------------------------------------
//
// Batches whose kernel has a closed-form simple profile (Fassett-Thomson or Martin-Parkes-Dunstan,
// neither complex, diffused nor tabulated), no rim smoothing, noise or texture, and whose records
// carry at most an ellipse and power-law outline harmonics (no rim table, marks, terraces, peaks,
// floor shift, upslope or datum) shape each crater by `fast_contribution`. It gives the
// reference's heights (craters.h:1028-1212 on that path) with fewer operations:
//   - the direction enters only through cos and sin of multiples of the angle, so they are
//     rotated by complex multiplication from (dx, dy) / r instead of atan2 then one cos per
//     harmonic: cos(k theta + phase) = A_k cos(k theta) - B_k sin(k theta), with
//     (A_k, B_k) = amplitude (cos phase, sin phase) prepared once per batch (`harmonics`);
//   - each harmonic's kept share, share^(k / 2), is a running product of sqrt(share).
// Both differ from the reference's float cosf / powf by a few ulp of terms of order 0.01.
struct FastKernel {
    uint32_t simple;  // kProfileFassettThomson or kProfileMartinParkesDunstan
    uint32_t rim;     // Fassett-Thomson rim mode
    float reachRadii;
};

__device__ __forceinline__ float fast_outline_scale(const float* __restrict__ harmonics,
                                                    const CraterRecord& c, float dx, float dy,
                                                    float distance, float share) {
    float c1 = 1.0f, s1 = 0.0f;  // the direction; angle 0 at the center, as KernelAngle
    if (distance > 0.0f) {
        c1 = dx / distance;
        s1 = dy / distance;
    }
    float scale = 1.0f;
    if (c.ellipticity != 1.0f) {
        // KernelEllipseScale (craters.h:737) with cos and sin of theta - heading by rotation.
        float sh, ch;
        sincosf(c.heading, &sh, &ch);
        const float cd = c1 * ch + s1 * sh;
        const float sd = s1 * ch - c1 * sh;
        const float along = sqrtf(c.ellipticity);
        const float across = 1.0f / along;
        const float u = cd / along;
        const float v = sd / across;
        scale = 1.0f / sqrtf(u * u + v * v);
    }
    float wobble = 1.0f;
    if (share > 0.0f && c.harmonicCount > 0u) {
        // (cm, sm) = (c1 + i s1)^m for the first harmonic's order m.
        float cm = 1.0f, sm = 0.0f;
        for (uint32_t i = 0; i < c.firstHarmonic; ++i) {
            const float t = cm * c1 - sm * s1;
            sm = cm * s1 + sm * c1;
            cm = t;
        }
        const bool partial = share < 1.0f;
        const float q = sqrtf(share);
        float kept = 1.0f;
        if (partial) {
            for (uint32_t i = 0; i < c.firstHarmonic; ++i) {
                kept *= q;
            }
        }
        // Two 4-byte loads per harmonic: a record's offset into the data may be odd.
        const float* h = harmonics + c.harmonicOffset;
        for (uint32_t n = 0; n < c.harmonicCount; ++n) {
            const float a = __ldg(h + 2u * n), b = __ldg(h + 2u * n + 1u);
            wobble += kept * (a * cm - b * sm);
            const float t = cm * c1 - sm * s1;
            sm = cm * s1 + sm * c1;
            cm = t;
            if (partial) {
                kept *= q;
            }
        }
    }
    return scale * wobble;
}

__device__ __forceinline__ float fast_contribution(const FastKernel& k,
                                                   const float* __restrict__ harmonics,
                                                   const CraterRecord& c, float dx, float dy,
                                                   bool& reached) {
    const float radius = 0.5f * c.diameter;
    float distance = sqrtf(dx * dx + dy * dy);
    if (c.ellipticity != 1.0f || c.harmonicCount > 0u) {
        const float share = outline_share(distance / radius) * worn_outline_share(c);
        distance /= fast_outline_scale(harmonics, c, dx, dy, distance, share);
    }
    reached = distance < k.reachRadii * radius;
    if (!reached) {
        return 0.0f;
    }
    float height;
    if (k.simple == kProfileMartinParkesDunstan) {
        height = mpd_height(distance, c.diameter, c.freshRim, c.currentDepth, c.currentRim);
    } else {
        height = ft_shape(distance / radius, k.rim, c.freshRim, c.currentDepth) * c.diameter;
    }
    return c.resolution * height;
}

// --- the plain path's lean craters -------------------------------------------------------------
//
// The plain binned kernel shapes most craters from a LeanCrater: what one crater's contribution
// reads, prepared once per crater (lean_crater) so that a (cell, crater) pair reads it in a few
// 16-byte shared-memory loads and spends no instruction on per-crater constants. It covers the
// closed-form simple profiles (Fassett-Thomson, Martin-Parkes-Dunstan), complex craters with their
// round central dome, ellipses and up to kLeanHarmonics power-law outline harmonics, under plain
// kernel options (no rim smoothing, noise, texture or diffusion). Each per-crater constant is the
// same float expression the per-pair path evaluates (complex_peak, the floor share, sincosf of
// the heading, ...), so it has the same bits. Per pair the outline's harmonics are summed by
// Horner's rule in the complex plane, sum_k (A_k + i B_k) (q e^{i theta})^k with q the square root
// of the kept share, which is the reference's sum of A_k cos(k theta + phase) share^(k/2) within
// a few float roundings. A crater with massif peaks is shaped here with its round dome, and the
// extras pass adds the massifs' difference from the dome in the bins the peak reaches; it also
// shapes the craters the lean path cannot (flag kLeanHeavy: tables, marks, terraces, floor
// shifts, upslopes, datums, more harmonics).
constexpr uint32_t kLeanHarmonics = 11;
constexpr uint32_t kLeanComplex = 2u;       // profile kind: 0 FT, 1 MPD, 2 complex
constexpr uint32_t kLeanOutline = 1u << 2;  // ellipse or harmonics
constexpr uint32_t kLeanEllipse = 1u << 3;
constexpr uint32_t kLeanHeavy = 1u << 4;    // the extras pass shapes it whole
constexpr uint32_t kLeanMassifs = 1u << 5;  // the extras pass adds its massif peak

struct __align__(16) LeanCrater {
    float x, xLow, y, yLow;
    float diameter, radius, resolution, reach;        // reach = reachRadii * radius
    float freshRim, currentDepth, currentRim, worn;   // worn = worn_outline_share
    float floorShare, peakBase, peakHeight, kept;     // complex craters
    float headingCos, headingSin, along, across;      // ellipse
    uint32_t flags;        // profile kind, kLean* bits, first harmonic << 8, count << 16
    uint32_t record;       // the crater's index in the batch
    float peakReach2;      // squared reach of its massif peak (kLeanMassifs)
    float ellipticity;
    float2 harmonics[kLeanHarmonics];  // (A cos phase, A sin phase)
    uint16_t tileX0, tileX1, tileY0, tileY1;  // the reference tiles its footprint window touches
    float cull;            // no cell beyond this distance (m) can be within its reach
    float invRadius;       // 1 / radius
    uint32_t pad[2];
};
static_assert(sizeof(LeanCrater) == 208, "LeanCrater must be a multiple of 16 bytes");
static_assert(offsetof(LeanCrater, harmonics) % 16 == 0 && kLeanHarmonics == 11,
              "the harmonics are read as five float4 and one float2");

// The lean form of record `c` under kernel `k` (harmonics from `data`), with its footprint's
// reference-tile box (x0, x1, y0, y1) and cull distance from the binning's count pass.
__device__ inline LeanCrater lean_crater(const CraterShapeKernel& k, const CraterRecord& c,
                                         const float* __restrict__ data, uint32_t index,
                                         int4 tiles, float cull) {
    LeanCrater l{};
    l.tileX0 = uint16_t(tiles.x);
    l.tileX1 = uint16_t(tiles.y);
    l.tileY0 = uint16_t(tiles.z);
    l.tileY1 = uint16_t(tiles.w);
    l.cull = cull;
    l.x = c.x;
    l.xLow = c.xLow;
    l.y = c.y;
    l.yLow = c.yLow;
    l.diameter = c.diameter;
    l.radius = 0.5f * c.diameter;
    l.invRadius = 1.0f / l.radius;
    l.resolution = c.resolution;
    l.reach = k.reachRadii * l.radius;
    l.freshRim = c.freshRim;
    l.currentDepth = c.currentDepth;
    l.currentRim = c.currentRim;
    l.worn = worn_outline_share(c);
    l.record = index;
    l.ellipticity = c.ellipticity;
    uint32_t flags = k.profile.simple == kProfileMartinParkesDunstan ? 1u : 0u;
    const bool complex = k.profile.complex == 1u && c.diameter >= k.profile.transitionDiameter;
    if (complex) {
        flags = kLeanComplex;
        const CraterProfileKernel& p = k.profile;
        l.floorShare = smin(
            0.9f, kilometer_law(p.floorCoefficient, p.floorExponent, c.diameter, false) /
                      c.diameter);
        const PeakSize size = complex_peak(p, c.diameter);
        l.peakBase = size.base;
        l.peakHeight = size.height;
        const State s{c.freshDepth, c.freshRim, c.currentDepth, c.currentRim};
        l.kept = kept_depth(s);
        if (c.peakCount > 0u) {
            flags |= kLeanMassifs;
            PeakSize scaled = size;
            scaled.base *= value(data, c.peakOffset + 5u);
            const float reach = TGB_PEAK_REACH * smax(size.base, scaled.base);
            l.peakReach2 = reach * reach;
        }
    }
    if (c.ellipticity != 1.0f) {
        flags |= kLeanEllipse;
        sincosf(c.heading, &l.headingSin, &l.headingCos);
        l.along = sqrtf(c.ellipticity);
        l.across = 1.0f / l.along;
    }
    if (c.ellipticity != 1.0f || c.harmonicCount > 0u) {
        flags |= kLeanOutline;
    }
    const bool heavy = c.tableCount > 0u || c.markCount > 0u || c.terraceCount > 0u ||
                       c.shiftX != 0.0f || c.shiftY != 0.0f || c.upslopeX != 0.0f ||
                       c.upslopeY != 0.0f || c.hasDatum == 1u ||
                       c.harmonicCount > kLeanHarmonics || c.firstHarmonic > 255u;
    if (heavy) {
        flags |= kLeanHeavy;
    } else {
        for (uint32_t h = 0; h < c.harmonicCount; ++h) {
            const float amplitude = value(data, c.harmonicOffset + 2u * h);
            const float phase = value(data, c.harmonicOffset + 2u * h + 1u);
            float sp, cp;
            sincosf(phase, &sp, &cp);
            l.harmonics[h] = make_float2(amplitude * cp, amplitude * sp);
        }
        flags |= (c.firstHarmonic << 8) | (c.harmonicCount << 16);
    }
    l.flags = flags;
    return l;
}

// The kernel's constants the lean path reads per pair, made once per launch: the complex
// exterior's value at its reach, edge = complexReachRadii^-ejectaExponent, and 1 / (1 - edge).
struct LeanKernel {
    float edge, fallScale;
};

__device__ __forceinline__ LeanKernel lean_kernel(const CraterShapeKernel& k) {
    const float edge = powf(k.profile.complexReachRadii, -k.profile.ejectaExponent);
    return LeanKernel{edge, 1.0f / (1.0f - edge)};
}

// What lean crater `l` adds at (dx, dy) from its center (resolution times the shaped relief, the
// round dome in place of massifs); `reached` is false beyond its reach. `shaped` receives the
// profile distance (after the outline), which the massif peak reads.
__device__ __forceinline__ float lean_contribution(const CraterShapeKernel& k,
                                                   const LeanKernel& lk, const LeanCrater& l,
                                                   float dx, float dy, bool& reached,
                                                   float& shaped) {
    const uint32_t flags = l.flags;
    const float d2 = dx * dx + dy * dy;
    // The distance and the direction from one reciprocal square root; the quotients below by
    // reciprocals made once per crater or by the fast divide. Each is within a few ulp of the
    // correctly rounded operation, far inside the heights' 1e-3 m tolerance and the cull
    // radius's 1e-5 relative margin.
    const float inv = d2 > 0.0f ? rsqrtf(d2) : 0.0f;
    float distance = d2 * inv;
    if (flags & kLeanOutline) {
        // KernelProfileDistance (craters.h:1028) with the outline's scale. The share is
        // smoothstep(distance / radius), exactly 1 from the rim out.
        const float share =
            (distance >= l.radius ? 1.0f : outline_share(distance * l.invRadius)) * l.worn;
        float c1 = 1.0f, s1 = 0.0f;  // the direction; angle 0 at the center, as KernelAngle
        if (distance > 0.0f) {
            c1 = dx * inv;
            s1 = dy * inv;
        }
        float scale = 1.0f;
        if (flags & kLeanEllipse) {
            const float cd = c1 * l.headingCos + s1 * l.headingSin;
            const float sd = s1 * l.headingCos - c1 * l.headingSin;
            const float u = cd * l.across;  // cd / along
            const float v = sd * l.along;   // sd / across
            scale = rsqrtf(u * u + v * v);
        }
        const uint32_t count = (flags >> 16) & 0xffu;
        if (share > 0.0f && count > 0u) {
            // w = q e^{i theta}, q = share^(1/2) (1 at full share). The harmonics past `count`
            // are zero, so Horner's rule runs over all kLeanHarmonics slots, unrolled: leading
            // zero terms leave the sum exactly as it is.
            const float q = share < 1.0f ? share * rsqrtf(share) : 1.0f;
            const float wr = q * c1, wi = q * s1;
            float pr = l.harmonics[kLeanHarmonics - 1u].x, pi = l.harmonics[kLeanHarmonics - 1u].y;
            // Harmonics 9 down to 0, two to a 16-byte load.
            const float4* pairs = reinterpret_cast<const float4*>(l.harmonics);
#pragma unroll
            for (int h = 4; h >= 0; --h) {
                const float4 v = pairs[h];  // harmonics 2h (x, y) and 2h + 1 (z, w)
                float t = pr * wr - pi * wi + v.z;
                pi = pr * wi + pi * wr + v.w;
                pr = t;
                t = pr * wr - pi * wi + v.x;
                pi = pr * wi + pi * wr + v.y;
                pr = t;
            }
            // times w^first
            uint32_t first = (flags >> 8) & 0xffu;
            if (first == 2u) {
                const float sr = wr * wr - wi * wi, si = 2.0f * wr * wi;  // w^2
                const float t = pr * sr - pi * si;
                pi = pr * si + pi * sr;
                pr = t;
            } else {
                for (; first > 0u; --first) {
                    const float t = pr * wr - pi * wi;
                    pi = pr * wi + pi * wr;
                    pr = t;
                }
            }
            scale *= 1.0f + pr;
        }
        distance = __fdividef(distance, scale);
    }
    shaped = distance;
    reached = distance < l.reach;
    if (!reached) {
        return 0.0f;
    }
    float height;
    const uint32_t kind = flags & 3u;
    if (kind == kLeanComplex) {
        // ComplexProfileHeight (craters.h:479) with its per-crater constants made once.
        const float x = distance * l.invRadius;
        const float depth = l.currentDepth * l.diameter;
        const float rim = l.currentRim * l.diameter;
        const CraterProfileKernel& p = k.profile;
        if (x >= 1.0f) {
            if (x >= p.complexReachRadii) {
                height = 0.0f;
            } else {
                const float fall = p.ejectaExponent == 3.0f ? __frcp_rn(x * x * x)
                                                            : powf(x, -p.ejectaExponent);
                height = rim * (fall - lk.edge) * lk.fallScale;
            }
        } else {
            height = rim - depth;
            if (x > l.floorShare) {
                const float t = (x - l.floorShare) / (1.0f - l.floorShare);
                height += depth * t * t;
            }
            height += l.kept * peak_dome(PeakSize{l.peakHeight, l.peakBase}, distance);
        }
    } else if (kind == 1u) {
        height = mpd_height(distance, l.diameter, l.freshRim, l.currentDepth, l.currentRim);
    } else {
        height = ft_shape(distance * l.invRadius, k.profile.rim, l.freshRim, l.currentDepth) *
                 l.diameter;
    }
    return l.resolution * height;
}

// The extras pass's contribution of crater `c` at (dx, dy): with kLeanHeavy its whole
// contribution (the general path); otherwise its massif peak's difference from the round dome
// the lean path gave it (KernelPeakRelief, craters.h:1161), times its resolution weight, 0 beyond
// the peak's reach.
static __device__ __noinline__ float extra_contribution(const CraterShapeKernel& k,
                                                        const float* data, const CraterRecord& c,
                                                        uint32_t flags, float dx, float dy,
                                                        bool& reached) {
    if (flags & kLeanHeavy) {
        const Contribution q = crater_contribution(k, data, c, dx, dy);
        reached = q.reached;
        return q.shaped;
    }
    const float distance = shifted_distance(data, c, dx, dy);
    reached = distance < k.reachRadii * (0.5f * c.diameter);
    if (!reached) {
        return 0.0f;
    }
    const State s{c.freshDepth, c.freshRim, c.currentDepth, c.currentRim};
    return c.resolution * peak_relief(k, data, c, s, distance, dx, dy);
}

}  // namespace crater
}  // namespace tgb
