// Crater populations drawn on the device (GenerateCraters on a plane:
// src/layers/craters/generation/population.cpp:381-441, SamplePoisson src/random/samplers.cpp:14-55,
// PowerLawSfd::Sample): one thread per generation cell of every band, in two passes (count, then
// write at the scanned offsets), so the output keeps the reference's order (band, cell row, cell
// column, draw).
//
// The draws are the reference's: Philox4x32-10 streams keyed as RandomStream keys them, the same
// double arithmetic (built with -fmad=false, as the host restatement is built with
// -ffp-contract=off), every per-band constant (exp(-mean), PTRS's logs, the SFD's terms) from the
// host's libm. Three device library calls remain: `pow` in the diameter's inversion, and `log` and
// `lgamma` in PTRS's acceptance test. The diameters may therefore differ from the host's in their
// last bits (counts, positions, ages and ids do not); a cell whose Poisson acceptance or keep
// decision lies within rounding of its threshold is flagged, and the host draws that cell instead,
// so counts and membership are always the reference's.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "population_plan.h"

using namespace tgb;
using namespace tgb::api;
using tgb::host::CraterBandPlan;
using tgb::host::HostCrater;

namespace {

constexpr uint32_t kCraterStream = 0x43524154u;    // streams.h:15-26
constexpr uint32_t kCraterAgeStream = 0x43524147u;
constexpr uint32_t kCraterIdStream = 0x43524944u;
constexpr int kMaxPoissonTries = 4096;             // PTRS accepts about 90 % of its proposals

struct Words4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ Words4 philox(Words4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = Words4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    }
    return c;
}

// RandomStream (stream.cpp:7-27): counter (a, b, c, block), 53-bit doubles from two words.
struct Stream {
    uint32_t k0, k1;
    Words4 counter, block;
    int used;
    __device__ Stream(uint32_t seed, uint32_t stream, uint32_t a, uint32_t b, uint32_t c)
        : k0(seed), k1(stream), counter{a, b, c, 0u}, block{0u, 0u, 0u, 0u}, used(4) {}
    __device__ uint32_t next_u32() {
        if (used == 4) {
            block = philox(counter, k0, k1);
            ++counter.w;
            used = 0;
        }
        const uint32_t v = used == 0 ? block.x : used == 1 ? block.y : used == 2 ? block.z : block.w;
        ++used;
        return v;
    }
    __device__ double next_double() {
        const uint64_t high = next_u32() >> 5u;
        const uint64_t low = next_u32() >> 6u;
        return double((high << 26u) | low) * 0x1p-53;
    }
};

struct DevicePlan {
    const CraterBandPlan* bands;
    uint32_t nBands;
    uint64_t cells;
    uint32_t seed;
    double c, lifetime, marginRadii;
    double region[4];
    double tolerance;  // relative width of a threshold within which a cell is flagged
    int32_t rootP, rootQ;  // the inversion's power as -rootQ / rootP (rootP a power of two), or 0
};

// A written diameter whose root lies near a rounding midpoint: its place and pow's argument.
struct RootFix {
    uint64_t at;
    double ratio;
};

// Double-double numbers (a value hi + lo, |lo| <= ulp(hi) / 2): Dekker's exact product by FMA
// and a renormalising sum, about 2^-104 relative per product.
struct Dd {
    double hi, lo;
};

__device__ __forceinline__ Dd dd_mul(Dd a, Dd b) {
    const double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e += a.hi * b.lo + a.lo * b.hi;
    const double s = p + e;
    return Dd{s, e - (s - p)};
}

__device__ __forceinline__ Dd dd_pow(Dd a, int n) {
    Dd r{1.0, 0.0};
    for (int k = 0; k < n; ++k) {
        r = dd_mul(r, a);
    }
    return r;
}

// The diameter of an inverse-CDF draw, x^(-q/p) for x = target / c (PowerLawSfd's inversion,
// std::pow(target / c, -1 / e) where the double -1 / e is exactly -q / p), correctly rounded: the
// device's pow gives a start within a few ulps, and each step compares the midpoints around the
// candidate with the root through m^p x^q = 1, in double-double (exact far beyond the decision
// below). The host's libm pow (glibc's: its exp step within 0.509 ulp, the log's error a few 1e-4
// ulp here) returns the correctly rounded root whenever the root lies more than about 0.01 ulp
// from a midpoint; a root within 0.05 ulp of one sets `ambiguous`, and the host's pow gives that
// diameter. With no -q / p (rootP 0) the device's pow stands and the diameter may differ from the
// host's in its last bits.
__device__ double sfd_root(double x, double inverseExponent, int p, int q, bool& ambiguous) {
    double y = pow(x, inverseExponent);
    if (p == 0) {
        return y;
    }
    const Dd xq = dd_pow(Dd{x, 0.0}, q);
    // m^p x^q - 1 for the double-double m.
    auto excess = [&](Dd m) {
        const Dd v = dd_mul(dd_pow(m, p), xq);
        return (v.hi - 1.0) + v.lo;
    };
    for (int step = 0; step < 8; ++step) {
        const double up = nextafter(y, INFINITY), down = nextafter(y, -INFINITY);
        const double halfUp = 0.5 * (up - y), halfDown = 0.5 * (down - y);
        const double above = excess(Dd{y, halfUp}), below = excess(Dd{y, halfDown});
        if (above > 0.0 && below < 0.0) {
            // The root is between the midpoints; its distance from each in ulps is about
            // |excess| y / p over the half-gap doubled.
            const double toUp = fabs(above) * y / (double(p) * 2.0 * halfUp);
            const double toDown = fabs(below) * y / (double(p) * -2.0 * halfDown);
            if (toUp < 0.05 || toDown < 0.05) {
                ambiguous = true;
            }
            return y;
        }
        y = above <= 0.0 ? up : down;
    }
    ambiguous = true;  // not bracketed in eight steps (never for pow's few-ulp start)
    return y;
}

__device__ __forceinline__ bool inside(const double* box, double x, double y) {
    return x >= box[0] && x < box[2] && y >= box[1] && y < box[3];
}

__device__ __forceinline__ bool inside_grown(const double* r, double m, double x, double y) {
    return x >= r[0] - m && x < r[2] + m && y >= r[1] - m && y < r[3] + m;
}

// SamplePoisson; `ambiguous` is set when an acceptance test lies within the tolerance.
__device__ uint64_t poisson(Stream& random, const CraterBandPlan& p, double tolerance,
                            bool& ambiguous) {
    if (p.mean == 0.0) {
        return 0;
    }
    if (p.mean < 10.0) {
        uint64_t count = 0;
        double product = random.next_double();
        while (product > p.limit) {
            ++count;
            product *= random.next_double();
        }
        return count;
    }
    for (int tries = 0; tries < kMaxPoissonTries; ++tries) {
        const double u = random.next_double() - 0.5;
        const double v = random.next_double();
        const double us = 0.5 - fabs(u);
        const double k = floor((2.0 * p.a / us + p.b) * u + p.mean + 0.43);
        if (us >= 0.07 && v <= p.vr) {
            return uint64_t(k);
        }
        if (k < 0.0 || (us < 0.013 && v > us)) {
            continue;
        }
        const double lhs = log(v) + p.logInverseAlpha - log(p.a / (us * us) + p.b);
        const double rhs = -p.mean + k * p.logMean - lgamma(k + 1.0);
        if (fabs(lhs - rhs) <= tolerance * (1.0 + fabs(lhs) + fabs(rhs))) {
            ambiguous = true;
        }
        if (lhs <= rhs) {
            return uint64_t(k);
        }
    }
    ambiguous = true;
    return 0;
}

// One cell's draws (GenerateCellCraters) and keep decisions; with `x` set, the kept craters are
// written from `at`. Returns the kept count.
__device__ uint32_t cell_pass(const DevicePlan& d, const CraterBandPlan& p, int32_t i, int32_t j,
                              bool& ambiguous, double* x, double* y, double* diameter,
                              double* age, uint64_t* id, uint64_t at, uint64_t capacity,
                              RootFix* fixes = nullptr, uint32_t* fixCount = nullptr) {
    Stream geometry(d.seed, kCraterStream, uint32_t(i), uint32_t(j), p.exponent);
    Stream ages(d.seed, kCraterAgeStream, uint32_t(i), uint32_t(j), p.exponent);
    const uint64_t count = poisson(geometry, p, d.tolerance, ambiguous);
    uint32_t kept = 0;
    for (uint64_t index = 0; index < count; ++index) {
        const double target = p.top - geometry.next_double() * p.count;
        // A root near a rounding midpoint leaves the cell's membership alone (the keep margin's
        // own slack covers a last-bit change); its diameter is the host's pow, patched in after
        // the write pass.
        bool nearMidpoint = false;
        const double ratio = target / d.c;
        double dia = sfd_root(ratio, p.inverseExponent, d.rootP, d.rootQ, nearMidpoint);
        dia = dia < p.low ? p.low : (p.high < dia ? p.high : dia);
        const double u = geometry.next_double();
        const double v = geometry.next_double();
        const double cx = (double(i) + u) * p.cellSize;
        const double cy = (double(j) + v) * p.cellSize;
        double a = ages.next_double() * d.lifetime;
        a = a < 0.0 ? 0.0 : (d.lifetime < a ? d.lifetime : a);
        if (!(cy >= p.outer[1] && cy <= p.outer[3])) {
            continue;
        }
        const bool inBand = dia >= p.low && dia <= p.high;
        if (inBand && !inside(p.outer, cx, cy)) {
            continue;
        }
        const double m = 0.5 * d.marginRadii * dia;
        bool keep = inside_grown(d.region, m, cx, cy);
        if (inBand && inside(p.inner, cx, cy)) {
            keep = true;
        } else {
            // The margin follows the diameter, whose last bits may differ from the host's.
            const double slack = d.tolerance * (m + 1.0);
            if (inside_grown(d.region, m - slack, cx, cy) !=
                inside_grown(d.region, m + slack, cx, cy)) {
                ambiguous = true;
            }
        }
        if (!keep) {
            continue;
        }
        if (x != nullptr && at + kept < capacity) {
            const Words4 w = philox(Words4{uint32_t(i), uint32_t(j), p.exponent, uint32_t(index)},
                                    d.seed, kCraterIdStream);
            const uint64_t n = at + kept;
            x[n] = cx;
            y[n] = cy;
            diameter[n] = dia;
            if (nearMidpoint && fixes != nullptr) {
                const uint32_t k = atomicAdd(fixCount, 1u);
                if (k < capacity) {
                    fixes[k] = RootFix{n, ratio};
                }
            }
            age[n] = a;
            id[n] = (uint64_t(w.x) << 32) | w.y;
        }
        ++kept;
    }
    return kept;
}

__device__ __forceinline__ const CraterBandPlan& band_of(const DevicePlan& d, uint64_t g,
                                                         int32_t& i, int32_t& j) {
    uint32_t b = 0;
    while (b + 1 < d.nBands && g >= d.bands[b + 1].firstCell) {
        ++b;
    }
    const CraterBandPlan& p = d.bands[b];
    const uint64_t local = g - p.firstCell;
    const uint64_t across = uint64_t(p.iMax - p.iMin + 1);
    i = p.iMin + int32_t(local % across);
    j = p.jMin + int32_t(local / across);
    return p;
}

__global__ void crater_count_cells_kernel(const DevicePlan d, uint32_t* __restrict__ counts,
                                          uint8_t* __restrict__ flags) {
    const uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= d.cells) {
        return;
    }
    int32_t i, j;
    const CraterBandPlan& p = band_of(d, g, i, j);
    bool ambiguous = false;
    counts[g] = cell_pass(d, p, i, j, ambiguous, nullptr, nullptr, nullptr, nullptr, nullptr, 0,
                          0);
    flags[g] = ambiguous ? 1u : 0u;
}

__global__ void crater_write_cells_kernel(const DevicePlan d, const uint64_t* __restrict__ offsets,
                                          const uint8_t* __restrict__ flags, double* x, double* y,
                                          double* diameter, double* age, uint64_t* id,
                                          uint64_t capacity, RootFix* fixes, uint32_t* fixCount) {
    const uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= d.cells || flags[g] != 0u) {
        return;
    }
    int32_t i, j;
    const CraterBandPlan& p = band_of(d, g, i, j);
    bool ambiguous = false;
    cell_pass(d, p, i, j, ambiguous, x, y, diameter, age, id, offsets[g], capacity, fixes,
              fixCount);
}

// The host's pow of the diameters whose roots lie near a rounding midpoint, to their places.
__global__ void patch_roots_kernel(const uint64_t* __restrict__ places,
                                   const double* __restrict__ values, uint32_t n,
                                   double* diameter) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        diameter[places[k]] = values[k];
    }
}

// The craters of host-drawn cells to their places in the outputs.
__global__ void scatter_hosted_kernel(const HostCrater* __restrict__ craters,
                                      const uint64_t* __restrict__ places, size_t n, double* x,
                                      double* y, double* diameter, double* age, uint64_t* id) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) {
        return;
    }
    const HostCrater c = craters[k];
    const uint64_t at = places[k];
    x[at] = c.x;
    y[at] = c.y;
    diameter[at] = c.diameter;
    age[at] = c.age;
    id[at] = c.id;
}

// A device allocation freed with its scope.
struct Scratch {
    void* ptr = nullptr;
    ~Scratch() {
        if (ptr != nullptr) {
            cudaFree(ptr);
        }
    }
    cudaError_t allocate(size_t bytes) {
        return cudaMalloc(&ptr, bytes > 0 ? bytes : 16);
    }
};

}  // namespace

extern "C" {

int tg_crater_generate_device(tg_device* d, const tg_crater_population* spec,
                              const double* region, double* x, double* y, double* diameter,
                              double* age, uint64_t* id, size_t capacity, size_t* count,
                              double tolerance, int memory, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    if (spec == nullptr || region == nullptr || count == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "population, region and count are required");
    }
    if (!(spec->min_diameter > 0.0) || !(spec->max_diameter > spec->min_diameter) ||
        !std::isfinite(spec->max_diameter) || !(spec->sfd_coefficient > 0.0) ||
        !(spec->sfd_exponent > 0.0) || !(spec->lifetime_gyr > 0.0) ||
        !(spec->cell_size_factor > 0.0) || !(region[2] >= region[0]) ||
        !(region[3] >= region[1])) {
        return fail(TG_ERROR_ARGUMENT, "population or region out of range");
    }
    if (!(tolerance >= 0.0) || !(tolerance < 1.0)) {
        return fail(TG_ERROR_ARGUMENT, "tolerance must be in [0, 1)");
    }
    if (tolerance == 0.0) {
        tolerance = 1e-9;  // far above the device's log, lgamma and pow errors
    }
    if (capacity > 0 && (x == nullptr || y == nullptr || diameter == nullptr || age == nullptr ||
                         id == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "output arrays are required with a capacity");
    }
    const std::vector<CraterBandPlan> plan = tgb::host::crater_plan(*spec, region);
    uint64_t cells = 0;
    for (const CraterBandPlan& p : plan) {
        if (p.iMax >= p.iMin && p.jMax >= p.jMin) {
            cells = p.firstCell + uint64_t(p.iMax - p.iMin + 1) * uint64_t(p.jMax - p.jMin + 1);
        }
    }
    *count = 0;
    if (cells == 0) {
        return TG_OK;
    }
    if (cells >= (uint64_t(1) << 32)) {
        return fail(TG_ERROR_UNSUPPORTED, "more than 2^32 generation cells");
    }
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    Scratch bands, counts, flags, offsets;
    TG_CUDA(bands.allocate(plan.size() * sizeof(CraterBandPlan)), "allocation");
    TG_CUDA(counts.allocate(cells * 4), "allocation");
    TG_CUDA(flags.allocate(cells), "allocation");
    TG_CUDA(offsets.allocate(cells * 8), "allocation");
    TG_CUDA(cudaMemcpyAsync(bands.ptr, plan.data(), plan.size() * sizeof(CraterBandPlan),
                            cudaMemcpyHostToDevice, s),
            "copy");
    DevicePlan dp{};
    dp.bands = static_cast<const CraterBandPlan*>(bands.ptr);
    dp.nBands = uint32_t(plan.size());
    dp.cells = cells;
    dp.seed = spec->seed;
    dp.c = spec->sfd_coefficient;
    dp.lifetime = spec->lifetime_gyr;
    dp.marginRadii = spec->margin_radii;
    std::memcpy(dp.region, region, 4 * sizeof(double));
    dp.tolerance = tolerance;
    // The inversion's power -1 / e as the double the host's pow takes: when that is -q / p with
    // p a power of two up to 16 and q up to 16 (e = 2, the craters' slope, gives -1 / 2), the
    // root is found correctly rounded.
    const double power = plan.empty() ? 0.0 : plan.front().inverseExponent;
    for (int p = 1; p <= 16; p *= 2) {
        const double q = -power * p;  // exact: a product by a power of two
        if (q >= 1.0 && q <= 16.0 && q == std::floor(q)) {
            dp.rootP = p;
            dp.rootQ = int32_t(q);
            break;
        }
    }
    const uint32_t blocks = uint32_t((cells + 127) / 128);
    crater_count_cells_kernel<<<blocks, 128, 0, s>>>(dp, static_cast<uint32_t*>(counts.ptr),
                                                     static_cast<uint8_t*>(flags.ptr));
    TG_CUDA(cudaGetLastError(), "count launch");
    std::vector<uint32_t> hc(cells);
    std::vector<uint8_t> hf(cells);
    TG_CUDA(cudaMemcpyAsync(hc.data(), counts.ptr, cells * 4, cudaMemcpyDeviceToHost, s), "copy");
    TG_CUDA(cudaMemcpyAsync(hf.data(), flags.ptr, cells, cudaMemcpyDeviceToHost, s), "copy");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    // The flagged cells on the host; then every cell's offset in draw order.
    std::vector<std::pair<uint64_t, std::vector<HostCrater>>> hosted;
    std::vector<uint64_t> off(cells);
    uint64_t total = 0;
    size_t b = 0;
    for (uint64_t g = 0; g < cells; ++g) {
        while (b + 1 < plan.size() && g >= plan[b + 1].firstCell) {
            ++b;
        }
        if (hf[g] != 0u) {
            const CraterBandPlan& p = plan[b];
            const uint64_t local = g - p.firstCell, across = uint64_t(p.iMax - p.iMin + 1);
            std::vector<HostCrater> list;
            tgb::host::cell_kept(*spec, region, p, p.iMin + int32_t(local % across),
                                 p.jMin + int32_t(local / across), list);
            hc[g] = uint32_t(list.size());
            hosted.emplace_back(g, std::move(list));
        }
        off[g] = total;
        total += hc[g];
    }
    *count = size_t(total);
    const uint64_t writable = std::min<uint64_t>(total, capacity);
    if (writable == 0) {
        return TG_OK;
    }
    // The outputs: the caller's device arrays, or device staging for host arrays.
    Scratch staged;
    double *dx = x, *dy = y, *dd = diameter, *da = age;
    uint64_t* di = id;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(staged.allocate(writable * 40), "allocation");
        dx = static_cast<double*>(staged.ptr);
        dy = dx + writable;
        dd = dy + writable;
        da = dd + writable;
        di = reinterpret_cast<uint64_t*>(da + writable);
    }
    TG_CUDA(cudaMemcpyAsync(offsets.ptr, off.data(), cells * 8, cudaMemcpyHostToDevice, s),
            "copy");
    // Room for every written crater's root fix (at most one each) and their count.
    Scratch fixes;
    TG_CUDA(fixes.allocate(writable * sizeof(RootFix) + 16), "allocation");
    uint32_t* fixCount = reinterpret_cast<uint32_t*>(static_cast<char*>(fixes.ptr) +
                                                     writable * sizeof(RootFix));
    TG_CUDA(cudaMemsetAsync(fixCount, 0, sizeof(uint32_t), s), "memset");
    crater_write_cells_kernel<<<blocks, 128, 0, s>>>(
        dp, static_cast<const uint64_t*>(offsets.ptr), static_cast<const uint8_t*>(flags.ptr),
        dx, dy, dd, da, di, writable, static_cast<RootFix*>(fixes.ptr), fixCount);
    TG_CUDA(cudaGetLastError(), "write launch");
    // The roots near a midpoint: the host's pow (the reference's libm) for each, patched in.
    uint32_t nFix = 0;
    TG_CUDA(cudaMemcpyAsync(&nFix, fixCount, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    Scratch patch;
    if (nFix > 0) {
        std::vector<RootFix> hostFixes(nFix);
        TG_CUDA(cudaMemcpyAsync(hostFixes.data(), fixes.ptr, nFix * sizeof(RootFix),
                                cudaMemcpyDeviceToHost, s),
                "copy");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        const double power = plan.front().inverseExponent;
        std::vector<uint64_t> places(nFix);
        std::vector<double> values(nFix);
        for (uint32_t k = 0; k < nFix; ++k) {
            places[k] = hostFixes[k].at;
            values[k] = std::pow(hostFixes[k].ratio, power);
        }
        TG_CUDA(patch.allocate(size_t(nFix) * 16), "allocation");
        uint64_t* dPlaces = static_cast<uint64_t*>(patch.ptr);
        double* dValues = reinterpret_cast<double*>(dPlaces + nFix);
        TG_CUDA(cudaMemcpyAsync(dPlaces, places.data(), size_t(nFix) * 8, cudaMemcpyHostToDevice,
                                s),
                "copy");
        TG_CUDA(cudaMemcpyAsync(dValues, values.data(), size_t(nFix) * 8, cudaMemcpyHostToDevice,
                                s),
                "copy");
        patch_roots_kernel<<<(nFix + 255) / 256, 256, 0, s>>>(dPlaces, dValues, nFix, dd);
        TG_CUDA(cudaGetLastError(), "patch launch");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");  // before the host vectors go
    }
    // The host-drawn cells' craters, gathered into one upload and scattered to their places.
    std::vector<HostCrater> flat;
    std::vector<uint64_t> places;
    for (const auto& [g, list] : hosted) {
        for (size_t k = 0; k < list.size() && off[g] + k < writable; ++k) {
            flat.push_back(list[k]);
            places.push_back(off[g] + k);
        }
    }
    Scratch hostedCraters, hostedPlaces;
    if (!flat.empty()) {
        TG_CUDA(hostedCraters.allocate(flat.size() * sizeof(HostCrater)), "allocation");
        TG_CUDA(hostedPlaces.allocate(places.size() * 8), "allocation");
        TG_CUDA(cudaMemcpyAsync(hostedCraters.ptr, flat.data(), flat.size() * sizeof(HostCrater),
                                cudaMemcpyHostToDevice, s),
                "copy");
        TG_CUDA(cudaMemcpyAsync(hostedPlaces.ptr, places.data(), places.size() * 8,
                                cudaMemcpyHostToDevice, s),
                "copy");
        scatter_hosted_kernel<<<uint32_t((flat.size() + 255) / 256), 256, 0, s>>>(
            static_cast<const HostCrater*>(hostedCraters.ptr),
            static_cast<const uint64_t*>(hostedPlaces.ptr), flat.size(), dx, dy, dd, da, di);
        TG_CUDA(cudaGetLastError(), "scatter launch");
    }
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(cudaMemcpyAsync(x, dx, writable * 8, cudaMemcpyDeviceToHost, s), "copy");
        TG_CUDA(cudaMemcpyAsync(y, dy, writable * 8, cudaMemcpyDeviceToHost, s), "copy");
        TG_CUDA(cudaMemcpyAsync(diameter, dd, writable * 8, cudaMemcpyDeviceToHost, s), "copy");
        TG_CUDA(cudaMemcpyAsync(age, da, writable * 8, cudaMemcpyDeviceToHost, s), "copy");
        TG_CUDA(cudaMemcpyAsync(id, di, writable * 8, cudaMemcpyDeviceToHost, s), "copy");
    }
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    return TG_OK;
}

}  // extern "C"
