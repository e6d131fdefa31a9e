// Device helpers shared by the binned kernels (craters.cu, boulders.cu, batch.cu): footprint
// windows on a grid, the dome relief, and the TMA bulk-copy / mbarrier staging primitives.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace tgb {
namespace binning {

constexpr uint32_t kSpinLimit = kWaitPolls;  // polls before a staged copy is given up on

__device__ __forceinline__ bool is_nodata(NoData nd, float h) {
    if (nd.mode == 1u) {
        return isnan(h);
    }
    return nd.mode != 0u && h == nd.value;
}

// `CraterOutline::MaxScale` (src/layers/craters/shaping/irregularity.cpp:229) from the record:
// sqrt(ellipticity) * (the largest 1 + table deviation, or 1 plus the harmonic amplitudes).
__device__ inline double max_outline_scale(const CraterRecord& r, const float* data) {
    double sum = 1.0;
    if (r.tableCount > 0u) {
        for (uint32_t n = 0; n < r.tableCount; ++n) {
            sum = fmax(sum, 1.0 + double(__ldg(data + r.tableOffset + n)));
        }
    } else {
        for (uint32_t n = 0; n < r.harmonicCount; ++n) {
            sum += fabs(double(__ldg(data + r.harmonicOffset + 2u * n)));
        }
    }
    return sqrt(double(r.ellipticity)) * sum;
}

__device__ __forceinline__ void world_to_pixel(const Grid& g, double x, double y, double& px,
                                               double& py) {
    // GeoTransform::WorldToPixel (include/terraingen/raster/geo_transform.h:70)
    const double det = g.pixelWidth * g.pixelHeight - g.rowRotation * g.colRotation;
    const double dx = x - g.originX;
    const double dy = y - g.originY;
    px = (dx * g.pixelHeight - dy * g.rowRotation) / det;
    py = (dy * g.pixelWidth - dx * g.colRotation) / det;
}

__device__ __forceinline__ int64_t clamp_index(double v, uint32_t limit) {
    // ClampIndex(v, limit + 1) (include/terraingen/util/bits.h:42)
    const double c = v < 0.0 ? 0.0 : (double(limit) < v ? double(limit) : v);
    return int64_t(c);
}

// The reference tile range a crater's footprint window touches; x0 > x1 when the window is
// empty. Also the radius beyond which a cell cannot be within the crater's reach, or +inf when
// marks, terraces or a floor shift stretch the profile distance past the outline's bound.
struct Footprint {
    int4 tiles;
    float cull;
};

// A crater's center and footprint reach in meters: from `footprints` (x, y, reach per record)
// when given, else from the record (center hi + lo, reach = outline stretch x reachRadii x
// radius); and its cull distance (see Footprint).
struct CraterReach {
    double x, y, reach;
    float cull;
};

__device__ inline CraterReach crater_reach(const CraterShapeKernel& k, const CraterRecord& r,
                                           const float* data, const double* footprints,
                                           uint32_t i) {
    CraterReach c;
    const double scale = max_outline_scale(r, data);
    if (footprints != nullptr) {
        c.x = footprints[3 * size_t(i)];
        c.y = footprints[3 * size_t(i) + 1];
        c.reach = footprints[3 * size_t(i) + 2];
    } else {
        c.x = double(r.x) + double(r.xLow);
        c.y = double(r.y) + double(r.yLow);
        c.reach = scale * double(k.reachRadii) * (0.5 * double(r.diameter));
    }
    const bool stretched = r.markCount > 0u || r.terraceCount > 0u || r.shiftX != 0.0f ||
                           r.shiftY != 0.0f;
    // A little slack over the bound: the profile distance is rounded in float.
    c.cull = stretched ? INFINITY
                       : float(scale * double(k.reachRadii) * (0.5 * double(r.diameter)) *
                               (1.0 + 1e-5)) + 1e-6f;
    return c;
}

// Whether a disk of `radius` around (x, y) meets the box (x0, y0, x1, y1).
__device__ __forceinline__ bool disk_meets_box(double x, double y, double radius,
                                               const double* box) {
    const double dx = fmax(fmax(box[0] - x, x - box[2]), 0.0);
    const double dy = fmax(fmax(box[1] - y, y - box[3]), 0.0);
    return dx * dx + dy * dy <= radius * radius;
}

// Whether the kernel's options add nothing beyond the profile and the outline: a closed-form
// simple profile (complex craters allowed), no diffusion tables, rim smoothing, noise, texture,
// ejecta or burial.
__host__ __device__ inline bool crater_options_plain(const CraterShapeKernel& k) {
    const CraterProfileKernel& p = k.profile;
    return (p.simple == kProfileFassettThomson || p.simple == kProfileMartinParkesDunstan) &&
           p.diffused == 0u && k.rimSigma == 0.0f && k.noiseAmplitude == 0.0f &&
           k.noiseRimAmplitude == 0.0f && k.wallStreaks == 0.0f && k.ejecta == 0.0f &&
           k.mantling == 0.0f;
}

// Whether a layer's binned entries fit the capacity the host gave them (the scan's total is in
// counts[bins]) and, for craters, none needs the ordered form (flag 1: a datum). The kernels after
// the scan do nothing otherwise; after the layer the host reads the total and the flags, grows the
// entries and runs the layer again (or reports the datum), so that binning needs no round trip to
// the host between the scan and the scatter.
__device__ __forceinline__ bool crater_bins_usable(const CraterBins& b) {
    return __ldg(b.counts + b.binsX * b.binsY) <= b.capacity && (b.total[1] & 1u) == 0u;
}
__device__ __forceinline__ bool boulder_bins_usable(const BoulderBins& b) {
    return __ldg(b.counts + b.binsX * b.binsY) <= b.capacity;
}

// Whether crater `r` shapes as a complex crater (FreshProfileHeight, craters.h:500).
__host__ __device__ inline bool crater_is_complex(const CraterShapeKernel& k,
                                                  const CraterRecord& r) {
    return k.profile.complex == 1u && r.diameter >= k.profile.transitionDiameter;
}

// Radii (of the outline-scaled profile distance) beyond which crater `r` adds nothing. The
// kernel's reach, except for a simple crater under a complex profile with plain options: the
// complex profile stretches every crater's reach to 3 radii (ComplexCraterProfile::ReachRadii),
// but a simple crater's relief is its simple profile's, exactly 0 beyond 1.5 radii
// (FassettThomsonShape) or 2 (MartinParkesDunstanHeight), and nothing else adds to it.
__host__ __device__ inline float crater_cull_radii(const CraterShapeKernel& k,
                                                   const CraterRecord& r) {
    if (k.profile.complex == 1u && !crater_is_complex(k, r) && crater_options_plain(k) &&
        r.peakCount == 0u && r.upslopeX == 0.0f && r.upslopeY == 0.0f && r.hasDatum == 0u) {
        const float simple = k.profile.simple == kProfileMartinParkesDunstan ? 2.0f : 1.5f;
        return simple < k.reachRadii ? simple : k.reachRadii;
    }
    return k.reachRadii;
}

__device__ inline Footprint crater_footprint(const CraterShapeKernel& k, const CraterRecord& r,
                                             const float* data, const double* footprints,
                                             uint32_t i, const Grid& g) {
    double x, y, reach;
    const double scale = max_outline_scale(r, data);
    if (footprints != nullptr) {
        x = footprints[3 * size_t(i)];
        y = footprints[3 * size_t(i) + 1];
        reach = footprints[3 * size_t(i) + 2];
    } else {
        x = double(r.x) + double(r.xLow);
        y = double(r.y) + double(r.yLow);
        reach = scale * double(k.reachRadii) * (0.5 * double(r.diameter));
    }
    // Surface::Expand on a plane, then MappedBounds of WorldToPixel (mapped_bounds.h).
    const double xs[2] = {x - reach, x + reach};
    const double ys[2] = {y - reach, y + reach};
    double minX = INFINITY, minY = INFINITY, maxX = -INFINITY, maxY = -INFINITY;
    for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 2; ++b) {
            double px, py;
            world_to_pixel(g, xs[a], ys[b], px, py);
            minX = fmin(minX, px);
            minY = fmin(minY, py);
            maxX = fmax(maxX, px);
            maxY = fmax(maxY, py);
        }
    }
    const int64_t c0 = clamp_index(floor(minX), g.width);
    const int64_t c1 = clamp_index(ceil(maxX), g.width);
    const int64_t r0 = clamp_index(floor(minY), g.height);
    const int64_t r1 = clamp_index(ceil(maxY), g.height);
    Footprint f;
    if (c0 >= c1 || r0 >= r1) {
        f.tiles = make_int4(1, 0, 1, 0);
    } else {
        f.tiles = make_int4(int(c0 / kRefTileCells), int((c1 - 1) / kRefTileCells),
                            int(r0 / kRefTileCells), int((r1 - 1) / kRefTileCells));
    }
    const bool stretched = r.markCount > 0u || r.terraceCount > 0u || r.shiftX != 0.0f ||
                           r.shiftY != 0.0f;
    // A little slack over the bound: the profile distance is rounded in float.
    f.cull = stretched ? INFINITY
                       : float(scale * double(crater_cull_radii(k, r)) *
                               (0.5 * double(r.diameter)) * (1.0 + 1e-5)) + 1e-6f;
    return f;
}

// Whether a record needs the general shaping path: anything beyond an ellipse and power-law
// harmonics (tables, marks, terraces, peaks, a floor shift, an upslope or a datum).
__device__ __forceinline__ bool crater_heavy(const CraterRecord& r) {
    return r.tableCount > 0u || r.markCount > 0u || r.terraceCount > 0u || r.peakCount > 0u ||
           r.shiftX != 0.0f || r.shiftY != 0.0f || r.upslopeX != 0.0f || r.upslopeY != 0.0f ||
           r.hasDatum == 1u;
}

// Whether the plain binned kernel's extras pass shapes crater `r` (crater_math.cuh
// `lean_crater`): a record the lean path cannot shape (tables, marks, terraces, a floor shift, an
// upslope, a datum, more than 11 outline harmonics).
__device__ __forceinline__ bool crater_needs_extras(const CraterShapeKernel& k,
                                                    const CraterRecord& r) {
    (void)k;
    return r.tableCount > 0u || r.markCount > 0u || r.terraceCount > 0u || r.shiftX != 0.0f ||
           r.shiftY != 0.0f || r.upslopeX != 0.0f || r.upslopeY != 0.0f || r.hasDatum == 1u ||
           r.harmonicCount > 11u || r.firstHarmonic > 255u;
}

// The pixel window of a box on the grid (PixelWindowIn, src/raster/cell_loops.cpp:21-28).
__device__ inline void window_of(const Grid& g, double minX, double minY, double maxX,
                                 double maxY, int& c0, int& c1, int& r0, int& r1) {
    const double det = g.pixelWidth * g.pixelHeight - g.rowRotation * g.colRotation;
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    const double xs[2] = {minX, maxX}, ys[2] = {minY, maxY};
    for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 2; ++b) {
            const double dx = xs[a] - g.originX, dy = ys[b] - g.originY;
            const double px = (dx * g.pixelHeight - dy * g.rowRotation) / det;
            const double py = (dy * g.pixelWidth - dx * g.colRotation) / det;
            lo[0] = fmin(lo[0], px);
            lo[1] = fmin(lo[1], py);
            hi[0] = fmax(hi[0], px);
            hi[1] = fmax(hi[1], py);
        }
    }
    auto clampi = [](double v, uint32_t limit) {
        return int(v < 0.0 ? 0.0 : (double(limit) < v ? double(limit) : v));
    };
    c0 = clampi(floor(lo[0]), g.width);
    c1 = clampi(ceil(hi[0]), g.width);
    r0 = clampi(floor(lo[1]), g.height);
    r1 = clampi(ceil(hi[1]), g.height);
}

// DomeHeight (boulder_relief.cpp:44): the dome's height at `distance` averaged over a band
// `width` wide, or at the point for a zero width.
__device__ __forceinline__ double dome(const BoulderEntry& b, double distance, double width) {
    const double radius = b.radius;
    if (!(width > 0.0)) {
        const double r2 = (distance * distance) / (radius * radius);
        return r2 < 1.0 ? b.exposed * sqrt(1.0 - r2) : 0.0;
    }
    auto area = [](double u) { return 0.5 * (u * sqrt(1.0 - u * u) + asin(u)); };
    const double low = fmin(fmax((distance - 0.5 * width) / radius, -1.0), 1.0);
    const double high = fmin(fmax((distance + 0.5 * width) / radius, -1.0), 1.0);
    if (!(high > low)) {
        return 0.0;
    }
    return b.exposed * (area(high) - area(low)) * radius / width;
}

// --- TMA bulk copy helpers (PTX ISA: cp.async.bulk, mbarrier) -------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return uint32_t(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// A bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global memory
// into this CTA's shared memory, completing on `bar`. The source is always this GPU's memory.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, "
        "1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return done != 0u;
}

// Waits for the barrier's phase, giving up after `limit` polls (returns false then).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase,
                                          uint32_t limit = kSpinLimit) {
    for (uint32_t spin = 0; spin < limit; ++spin) {
        if (mbar_try_wait(bar, phase)) {
            return true;
        }
    }
    return false;
}

}  // namespace binning
}  // namespace tgb
