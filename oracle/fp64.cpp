// oracle/fp64.cpp - test infrastructure only, never linked into the product.
//
// The FP64 oracle of the crater and boulder layers: the reference's own crater kernel header
// (include/terraingen/layers/kernels/craters.h, with the noise headers it includes) compiled with
// every `float` spelled `double`, so its shaping functions (profiles, outlines, terraces, massif
// peaks, noise, texture) run in double with the reference's operation order; only the float
// literals keep their float values. Built from the reference checkout by oracle/Makefile into
// oracle/_ref/libtgfp64.so; nothing of the reference is copied here.
//
// Inputs are the float std430 bytes a crater layer hands its kernel (the shape kernel, the
// records in apply order, the float data), widened field by field to the double build's structs;
// a crater's center is its split float pair summed in double. Cell positions are exact doubles.
// The boulder layer's dome (DomeHeight, src/layers/boulders/boulder_relief.cpp:44-57) is already
// FP64 in the reference; it is restated here so that the composite stays in double (no float
// rounding of the heights between layers).

// Every standard header the included reference headers use comes first, so the spelling change
// below reaches only the reference's own declarations.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "terraingen/util/span.h"

namespace terraingen {
// The header mixes float literals with (now double) values in min / max / clamp, which the
// standard templates cannot deduce; these take both as double.
inline double min(double a, double b) {
    return a < b ? a : b;
}
inline double max(double a, double b) {
    return a < b ? b : a;
}
inline double clamp(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}
}  // namespace terraingen

#define float double
#define static_assert(...)
#include "terraingen/layers/kernels/craters.h"
#undef static_assert
#undef float

namespace {

using terraingen::CraterProfileKind;
using terraingen::CraterRecord;
using terraingen::CraterShapeKernel;

// Reads 4-byte std430 words in field order into the double build's structs.
struct Words {
    const uint8_t* at;
    float f() {
        float v;
        std::memcpy(&v, at, 4);
        at += 4;
        return v;
    }
    uint32_t u() {
        uint32_t v;
        std::memcpy(&v, at, 4);
        at += 4;
        return v;
    }
    int32_t i() {
        int32_t v;
        std::memcpy(&v, at, 4);
        at += 4;
        return v;
    }
};

CraterShapeKernel widen_kernel(const void* bytes) {
    Words w{static_cast<const uint8_t*>(bytes)};
    CraterShapeKernel k;
    auto& p = k.profile;
    p.simple = static_cast<CraterProfileKind>(w.u());
    p.rim = w.u();
    p.complex = w.u();
    p.diffused = w.u();
    p.transitionDiameter = w.f();
    p.floorCoefficient = w.f();
    p.floorExponent = w.f();
    p.peakHeightCoefficient = w.f();
    p.peakHeightExponent = w.f();
    p.peakWidthCoefficient = w.f();
    p.peakWidthExponent = w.f();
    p.peakFromVolume = w.u();
    p.peakFitMaxDiameter = w.f();
    p.ejectaExponent = w.f();
    p.complexReachRadii = w.f();
    p.tableExtent = w.f();
    p.tableCells = w.u();
    p.agesOffset = w.u();
    p.ageCount = w.u();
    k.reachRadii = w.f();
    k.profileReachRadii = w.f();
    k.blendStart = w.f();
    k.blendEnd = w.f();
    k.blendShape = w.u();
    k.interiorReplacement = w.f();
    k.replaceStart = w.f();
    k.replaceEnd = w.f();
    k.mantling = w.f();
    k.ejectaReachRadii = w.f();
    k.rimSigma = w.f();
    k.rimInner = w.f();
    k.rimOuter = w.f();
    k.rimStrength = w.f();
    k.rimShape = w.u();
    k.noiseAmplitude = w.f();
    k.noiseWavelength = w.f();
    k.noiseOctaves = w.i();
    k.noiseGain = w.f();
    k.noiseRimAmplitude = w.f();
    k.noiseRimWavelength = w.f();
    k.noiseRimInner = w.f();
    k.noiseRimOuter = w.f();
    k.wallStreaks = w.f();
    k.wallStreakWidth = w.f();
    k.ejecta = w.f();
    k.ejectaLineation = w.f();
    k.minFreshness = w.f();
    return k;
}

CraterRecord widen_record(const void* bytes) {
    Words w{static_cast<const uint8_t*>(bytes)};
    CraterRecord r;
    r.x = w.f();
    r.y = w.f();
    r.diameter = w.f();
    r.resolution = w.f();
    r.freshDepth = w.f();
    r.freshRim = w.f();
    r.currentDepth = w.f();
    r.currentRim = w.f();
    r.diffusion = w.f();
    r.ellipticity = w.f();
    r.heading = w.f();
    r.firstHarmonic = w.u();
    r.harmonicCount = w.u();
    r.harmonicOffset = w.u();
    r.tableCount = w.u();
    r.tableOffset = w.u();
    r.profileOffset = w.u();
    r.hasDatum = w.u();
    r.datumA = w.f();
    r.datumB = w.f();
    r.datumC = w.f();
    r.noiseKey = w.u();
    r.textureKey = w.u();
    r.markCount = w.u();
    r.markOffset = w.u();
    r.shiftX = w.f();
    r.shiftY = w.f();
    r.upslopeX = w.f();
    r.upslopeY = w.f();
    r.terraceCount = w.u();
    r.terraceOffset = w.u();
    r.peakCount = w.u();
    r.peakOffset = w.u();
    r.replace = w.u();
    r.xLow = w.f();
    r.yLow = w.f();
    return r;
}

}  // namespace

extern "C" {

// The crater layer in FP64 on a north-up grid (x0, y0 its top-left corner, square cells of
// `pixel` m): each record in order, with ApplyCraterKernel (craters.h:1186), on every cell whose
// center lies within its footprint reach (`footprints`: x, y, reach per record, as
// tg_crater_batch gives them; beyond it the kernel leaves the height unchanged). `heights`
// (width x height doubles, row 0 north) holds the heights before the layer and receives those
// after it. Returns 0.
int f64_craters(const void* kernel, const void* records, size_t n, const float* data,
                size_t n_data, const double* footprints, uint32_t width, uint32_t height,
                double x0, double y0, double pixel, double* heights) {
    const CraterShapeKernel k = widen_kernel(kernel);
    std::vector<double> values(data, data + n_data);
    const uint8_t* rec = static_cast<const uint8_t*>(records);
    for (size_t i = 0; i < n; ++i) {
        const CraterRecord c = widen_record(rec + 144 * i);
        const double cx = c.x + c.xLow, cy = c.y + c.yLow;
        const double reach = footprints[3 * i + 2] + 2.0 * pixel;
        const long c0 = std::max(0L, long(std::floor((cx - reach - x0) / pixel)));
        const long c1 = std::min(long(width) - 1, long(std::ceil((cx + reach - x0) / pixel)));
        const long r0 = std::max(0L, long(std::floor((y0 - cy - reach) / pixel)));
        const long r1 = std::min(long(height) - 1, long(std::ceil((y0 - cy + reach) / pixel)));
        for (long row = r0; row <= r1; ++row) {
            const double py = y0 - (double(row) + 0.5) * pixel;
            for (long col = c0; col <= c1; ++col) {
                const double px = x0 + (double(col) + 0.5) * pixel;
                double& h = heights[size_t(row) * width + size_t(col)];
                h = terraingen::ApplyCraterKernel(k, terraingen::CraterData{values.data()}, c, h,
                                                  px - cx, py - cy);
            }
        }
    }
    return 0;
}

// The boulder layer in FP64 (BoulderLayer::ApplySamples with dome relief,
// src/layers/boulders/boulder_relief.cpp:244-275, 426-439): each boulder (x, y, diameter,
// exposed height, resolution weight) raises the cells of its box to at least the height before
// the layer plus weight x its dome averaged over a sample `sample_width` wide (DomeHeight,
// :44-57). `heights` as for f64_craters.
void f64_boulders(const double* boulders, size_t n, double sample_width, uint32_t width,
                  uint32_t height, double x0, double y0, double pixel, double* heights) {
    const std::vector<double> base(heights, heights + size_t(width) * height);
    auto area = [](double u) { return 0.5 * (u * std::sqrt(1.0 - u * u) + std::asin(u)); };
    for (size_t i = 0; i < n; ++i) {
        const double* b = boulders + 5 * i;
        const double radius = 0.5 * b[2];
        const double reach = 0.5 * (b[2] + sample_width);
        const long c0 = std::max(0L, long(std::floor((b[0] - reach - x0) / pixel)));
        const long c1 = std::min(long(width) - 1, long(std::ceil((b[0] + reach - x0) / pixel)));
        const long r0 = std::max(0L, long(std::floor((y0 - b[1] - reach) / pixel)));
        const long r1 = std::min(long(height) - 1, long(std::ceil((y0 - b[1] + reach) / pixel)));
        for (long row = r0; row <= r1; ++row) {
            const double py = y0 - (double(row) + 0.5) * pixel;
            for (long col = c0; col <= c1; ++col) {
                const double px = x0 + (double(col) + 0.5) * pixel;
                const double distance = std::hypot(px - b[0], py - b[1]);
                double dome = 0.0;
                if (!(sample_width > 0.0)) {
                    const double r2 = distance * distance / (radius * radius);
                    dome = r2 < 1.0 ? b[3] * std::sqrt(1.0 - r2) : 0.0;
                } else {
                    const double lo = std::clamp((distance - 0.5 * sample_width) / radius, -1.0, 1.0);
                    const double hi = std::clamp((distance + 0.5 * sample_width) / radius, -1.0, 1.0);
                    dome = hi > lo ? b[3] * (area(hi) - area(lo)) * radius / sample_width : 0.0;
                }
                const double relief = std::max(dome, 0.0);
                if (relief > 0.0) {
                    const size_t at = size_t(row) * width + size_t(col);
                    heights[at] = std::max(heights[at], base[at] + b[4] * relief);
                }
            }
        }
    }
}

}  // extern "C"
