// Crater kernel records built on the device: CraterApplyOrder and MakeCraterKernelBatch's
// per-crater work (src/layers/craters/shaping/crater_kernel.cpp:187-622, irregularity.cpp:
// 165-300, apply_options.cpp:96) for a batch whose population, candidates, wall terraces and
// massif peaks the host has made (population.cpp record_plan). The apply order (age descending,
// then diameter descending, id, draw index) is three stable radix sorts of 64-bit keys, least
// significant first, from the draw order. Then one thread per crater, in apply order, draws its
// outline (Philox4x32-10 on its irregularity stream), takes its exact footprint and writes its
// record, its harmonics, its extras and its footprint at offsets an exclusive scan gives, so the
// batch is tg_crater_batch's byte for byte: every operation here is IEEE double arithmetic the
// host does in the same order (this unit is compiled with -fmad=false), and the only libm work of
// a record, the terraces' and peaks' trigonometry, stays on the host.

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "api_internal.h"
#include "crater_records.h"
#include "layouts.h"
#include "noise_math.cuh"

namespace tgb {
namespace {

constexpr uint32_t kIrregularityStream = 0x49525247u;  // streams.h: kCraterIrregularityStream
constexpr int kOutlineHarmonics = 11;                   // harmonics 2..12

struct Words {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ Words philox10(Words c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = Words{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    }
    return c;
}

// A keyed stream's doubles in order (Stream::next_double: 27 and 26 bits of two words).
struct DeviceStream {
    Words counter, block;
    uint32_t k0, k1;
    int used;

    __device__ DeviceStream(uint32_t seed, uint32_t stream, uint32_t a, uint32_t b)
        : counter{a, b, 0u, 0u}, block{0u, 0u, 0u, 0u}, k0(seed), k1(stream), used(4) {}

    __device__ uint32_t next_u32() {
        if (used == 4) {
            block = philox10(counter, k0, k1);
            ++counter.w;
            used = 0;
        }
        const uint32_t v = used == 0 ? block.x : used == 1 ? block.y : used == 2 ? block.z
                                                                        : block.w;
        ++used;
        return v;
    }
    __device__ double next_double() {
        const uint64_t high = next_u32() >> 5u;
        const uint64_t low = next_u32() >> 6u;
        return double((high << 26u) | low) * 0x1p-53;
    }
};

struct DeviceOutline {
    double ellipticity, heading;
    double amplitudes[kOutlineHarmonics], phases[kOutlineHarmonics];
    int harmonics, firstHarmonic;
};

// IrregularOutline with the default irregularity, as the host's irregular_outline.
__device__ void outline_of(const RecordConstants& k, uint64_t id, DeviceOutline& o) {
    o.ellipticity = 1.0;
    o.heading = 0.0;
    o.harmonics = 0;
    o.firstHarmonic = 2;
    if (k.irregular == 0u) {
        return;
    }
    DeviceStream random(k.irregularitySeed, kIrregularityStream, uint32_t(id), uint32_t(id >> 32));
    double d[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        d[i] = random.next_double();
    }
    const double rough = d[0], elongated = d[1], r1 = d[2], e1 = d[6], h = d[8];
    if (elongated < 0.054) {
        o.ellipticity = 1.1 + (1.5 - 1.1) * e1;
        o.heading = 3.14159265358979323846 * h;
    }
    if (rough < 1.0) {
        const double roughness = 0.01 + (0.03 - 0.01) * r1;
        const double norm = roughness * k.outlineScale;
        if (roughness > 0.0) {
            for (int n = 0; n < kOutlineHarmonics; ++n) {
                o.amplitudes[n] = norm * k.outlinePower[n];
                o.phases[n] = 2.0 * 3.14159265358979323846 * random.next_double();
            }
            o.harmonics = kOutlineHarmonics;
        }
    }
}

__device__ __forceinline__ double clamp(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);  // std::clamp
}

// 1 - Falloff(D / spacing, 2, 4, Smoothstep) (src/layers/fade.cpp:18-52).
__device__ double resolution_weight(double diameter, double spacing) {
    const double x = diameter / spacing;
    double f;
    if (x <= 2.0) {
        f = 1.0;
    } else if (x >= 4.0) {
        f = 0.0;
    } else {
        double t = clamp((x - 2.0) / (4.0 - 2.0), 0.0, 1.0);
        f = 1.0 - t * t * (3.0 - 2.0 * t);
    }
    return 1.0 - f;
}

// Whether the footprint box of half-width `reach` around (x, y) holds a cell of the grid
// (Surface::Expand, MappedBounds of WorldToPixel over the box's corners, ClampIndex).
__device__ bool footprint_cells(const RecordConstants& k, double x, double y, double reach) {
    const double det = k.pixelWidth * k.pixelHeight - k.rowRotation * k.colRotation;
    double minX = INFINITY, minY = INFINITY, maxX = -INFINITY, maxY = -INFINITY;
    const double wxs[2] = {x - reach, x + reach};
    const double wys[2] = {y - reach, y + reach};
#pragma unroll
    for (int a = 0; a < 2; ++a) {
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const double dx = wxs[a] - k.originX;
            const double dy = wys[b] - k.originY;
            const double px = (dx * k.pixelHeight - dy * k.rowRotation) / det;
            const double py = (dy * k.pixelWidth - dx * k.colRotation) / det;
            minX = fmin(minX, px);
            minY = fmin(minY, py);
            maxX = fmax(maxX, px);
            maxY = fmax(maxY, py);
        }
    }
    const double c0 = clamp(floor(minX), 0.0, k.width);
    const double c1 = clamp(ceil(maxX), 0.0, k.width);
    const double r0 = clamp(floor(minY), 0.0, k.height);
    const double r1 = clamp(ceil(maxY), 0.0, k.height);
    return uint64_t(c0) < uint64_t(c1) && uint64_t(r0) < uint64_t(r1);
}

// The crater's outline, resolution weight and exact reach; false when it gives no record.
__device__ bool crater_reach(const RecordConstants& k, const RecordCrater& c, DeviceOutline& o,
                             double& resolution, double& reach) {
    resolution = resolution_weight(c.diameter, k.spacing);
    if (resolution == 0.0) {
        return false;
    }
    outline_of(k, c.id, o);
    double scale = 1.0;
    for (int n = 0; n < o.harmonics; ++n) {
        scale += fabs(o.amplitudes[n]);
    }
    scale *= sqrt(o.ellipticity);
    reach = scale * k.reachRadii * (0.5 * c.diameter);
    return footprint_cells(k, c.x, c.y, reach);
}

__device__ __forceinline__ uint32_t crater_key(uint64_t id, uint32_t seed) {  // hash.h:68
    return noise::pcg(uint32_t(id) ^ noise::pcg(uint32_t(id >> 32u) ^ seed));
}

// The apply order's sort keys, as unsigned integers in ascending order: `field` 0 the id, 1 the
// diameter descending, 2 the age descending (both positive doubles, whose bits order as their
// values, complemented), read through the order so far (`order`; null: the draw order, which
// `orderOut` then receives).
__global__ void order_keys_kernel(const RecordCrater* __restrict__ craters, uint32_t n,
                                  const uint32_t* __restrict__ order, int field,
                                  uint64_t* __restrict__ keys, uint32_t* __restrict__ orderOut) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint32_t at = order != nullptr ? order[i] : i;
    if (order == nullptr) {
        orderOut[i] = i;
    }
    const RecordCrater& c = craters[at];
    keys[i] = field == 0   ? c.id
              : field == 1 ? ~uint64_t(__double_as_longlong(c.diameter))
                           : ~uint64_t(__double_as_longlong(c.age));
}

// Pass 1: each crater's record (1 or 0) and data floats, in apply order.
__global__ void record_count_kernel(const RecordCrater* __restrict__ craters,
                                    const uint32_t* __restrict__ order, uint32_t n,
                                    const RecordConstants k, uint32_t* __restrict__ records,
                                    uint32_t* __restrict__ floats) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const RecordCrater c = craters[order[i]];
    DeviceOutline o;
    double resolution, reach;
    const bool kept = crater_reach(k, c, o, resolution, reach);
    records[i] = kept ? 1u : 0u;
    floats[i] = kept ? uint32_t(2 * o.harmonics) + c.extraFloats : 0u;
}

// Pass 2: the records, data and footprints at the scanned offsets (nothing past a capacity).
__global__ void record_write_kernel(const RecordCrater* __restrict__ craters,
                                    const uint32_t* __restrict__ order, uint32_t n,
                                    const RecordConstants k, const float* __restrict__ extras,
                                    const uint32_t* __restrict__ recordAt,
                                    const uint32_t* __restrict__ dataAt, size_t recordCapacity,
                                    size_t dataCapacity, CraterRecord* __restrict__ records,
                                    float* __restrict__ data, double* __restrict__ footprints) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || recordAt[i + 1] == recordAt[i]) {
        return;
    }
    const RecordCrater c = craters[order[i]];
    DeviceOutline o;
    double resolution, reach;
    crater_reach(k, c, o, resolution, reach);
    const uint32_t at = recordAt[i];
    const uint32_t base = dataAt[i];
    const uint32_t harmonicFloats = uint32_t(2 * o.harmonics);
    if (data != nullptr && size_t(base) + harmonicFloats + c.extraFloats <= dataCapacity) {
        for (int n = 0; n < o.harmonics; ++n) {
            data[base + 2 * n] = float(o.amplitudes[n]);
            data[base + 2 * n + 1] = float(o.phases[n]);
        }
        for (uint32_t e = 0; e < c.extraFloats; ++e) {
            data[base + harmonicFloats + e] = extras[c.extraOffset + e];
        }
    }
    if (footprints != nullptr && at < recordCapacity) {
        footprints[3 * size_t(at)] = c.x;
        footprints[3 * size_t(at) + 1] = c.y;
        footprints[3 * size_t(at) + 2] = reach;
    }
    if (records == nullptr || at >= recordCapacity) {
        return;
    }
    CraterRecord r;
    memset(&r, 0, sizeof(r));
    r.diameter = float(c.diameter);
    r.freshDepth = float(k.freshDepth);
    r.freshRim = float(k.freshRim);
    r.currentDepth = float(c.erosion * k.freshDepth);
    r.currentRim = float(c.erosion * k.freshRim);
    r.resolution = float(resolution);
    r.noiseKey = crater_key(c.id, k.noiseSeed);
    r.textureKey = crater_key(c.id, k.textureKeySeed);
    r.x = float(c.x);
    r.xLow = float(c.x - double(r.x));
    r.y = float(c.y);
    r.yLow = float(c.y - double(r.y));
    r.ellipticity = float(o.ellipticity);
    r.heading = float(o.heading);
    r.harmonicOffset = base;
    r.firstHarmonic = uint32_t(o.firstHarmonic);
    r.harmonicCount = uint32_t(o.harmonics);
    r.tableOffset = base + harmonicFloats;
    r.markOffset = base + harmonicFloats;
    r.terraceCount = c.terraceCount;
    r.terraceOffset = c.terraceCount > 0u ? base + harmonicFloats : 0u;
    r.peakCount = c.peakCount;
    r.peakOffset = c.peakCount > 0u ? base + harmonicFloats + c.terraceFloats : 0u;
    records[at] = r;
}

// The caller's page-locked staging for the plan, grown as needed and kept by the device.
int stage(tg_device* d, size_t bytes) {
    if (bytes <= d->recordStageBytes) {
        return TG_OK;
    }
    if (d->recordStage != nullptr) {
        cudaFreeHost(d->recordStage);
        d->recordStage = nullptr;
        d->recordStageBytes = 0;
    }
    const size_t size = bytes + bytes / 2;
    TG_CUDA(cudaMallocHost(&d->recordStage, size), "page-locked allocation");
    d->recordStageBytes = size;
    return TG_OK;
}

}  // namespace
}  // namespace tgb

using namespace tgb;
using namespace tgb::api;

extern "C" {

int tg_crater_batch_device(tg_device* d, const tg_crater_population* spec,
                           const tg_crater_shaping* shaping, const tg_grid* grid, void* kernel,
                           void* records, size_t record_capacity, float* data,
                           size_t data_capacity, double* footprints, size_t* n_records,
                           size_t* n_data, size_t* staged_bytes, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    if (spec == nullptr || shaping == nullptr || grid == nullptr || n_records == nullptr ||
        n_data == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "population, shaping, grid and counts are required");
    }
    // The device is held for the whole call, its host part included: the plan is written
    // straight into the device's page-locked staging.
    std::lock_guard<std::mutex> lock(d->mutex);
    TG_CUDA(cudaSetDevice(d->ordinal), "set device");
    // The population, the apply order, the terraces and peaks on the host threads; the craters
    // in apply order into the staging, the extras after them below.
    static thread_local std::vector<float> extras;
    RecordConstants k{};
    size_t n = 0;
    int staged = TG_OK;
    const auto place = [&](size_t count) -> RecordCrater* {
        staged = stage(d, count * sizeof(RecordCrater) + (size_t(1) << 20));
        return staged == TG_OK ? static_cast<RecordCrater*>(d->recordStage) : nullptr;
    };
    if (int st = host::record_plan(*spec, *shaping, *grid, kernel, k, place, n, extras)) {
        if (staged != TG_OK) {
            return staged;
        }
        return fail(st, st == TG_ERROR_UNSUPPORTED
                            ? "rotated or south-up grids, or more than 2^32 craters or floats"
                            : "population or shaping out of range");
    }
    if (n >= 0xffffffffu) {
        return fail(TG_ERROR_UNSUPPORTED, "more than 2^32 - 1 craters");
    }
    const cudaStream_t s = stream != nullptr ? static_cast<cudaStream_t>(stream) : d->stream;
    *n_records = 0;
    *n_data = 1;
    if (staged_bytes != nullptr) {
        *staged_bytes = 0;
    }
    const bool query = records == nullptr && data == nullptr && footprints == nullptr;
    if (n == 0) {
        if (data != nullptr && data_capacity >= 1) {
            TG_CUDA(cudaMemsetAsync(data, 0, sizeof(float), s), "clear");
            TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        }
        return data != nullptr && data_capacity < 1
                   ? fail(TG_ERROR_ARGUMENT, "data capacity below the batch's 1 float")
                   : TG_OK;
    }
    // The plan crosses once, through the device's page-locked staging: the craters are there,
    // the extras follow them (the staging grown, the craters kept, when they do not fit).
    const size_t craterBytes = n * sizeof(RecordCrater);
    const size_t extraBytes = std::max<size_t>(extras.size(), 1) * sizeof(float);
    if (craterBytes + extraBytes > d->recordStageBytes) {
        std::vector<char> keep(static_cast<char*>(d->recordStage),
                               static_cast<char*>(d->recordStage) + craterBytes);
        if (int st = stage(d, craterBytes + extraBytes)) {
            return st;
        }
        std::memcpy(d->recordStage, keep.data(), craterBytes);
    }
    if (!extras.empty()) {
        std::memcpy(static_cast<char*>(d->recordStage) + craterBytes, extras.data(),
                    extras.size() * sizeof(float));
    }
    const uint32_t scanWords = uint32_t(scan_scratch_words(uint32_t(n)));
    TG_CUDA(d->slots[kRecordCraters].reserve(craterBytes + extraBytes), "allocation");
    TG_CUDA(d->slots[kRecordCounts].reserve(2 * (n + 1) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kScan].reserve(size_t(scanWords) * sizeof(uint32_t)), "allocation");
    auto* dCraters = static_cast<RecordCrater*>(d->slots[kRecordCraters].ptr);
    auto* dExtras = reinterpret_cast<float*>(static_cast<char*>(d->slots[kRecordCraters].ptr) +
                                             craterBytes);
    auto* recordAt = static_cast<uint32_t*>(d->slots[kRecordCounts].ptr);
    uint32_t* dataAt = recordAt + (n + 1);
    TG_CUDA(cudaMemcpyAsync(dCraters, d->recordStage, craterBytes + extraBytes,
                            cudaMemcpyHostToDevice, s),
            "copy");
    if (staged_bytes != nullptr) {
        *staged_bytes = craterBytes + extraBytes;
    }
    const uint32_t blocks = uint32_t((n + 255) / 256);
    // CraterApplyOrder: stable sorts by the id, then the diameter descending, then the age
    // descending, from the draw order (the last key of the comparison).
    size_t sortBytes = 0;
    TG_CUDA(cub::DeviceRadixSort::SortPairs(
                nullptr, sortBytes, static_cast<const uint64_t*>(nullptr),
                static_cast<uint64_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                static_cast<uint32_t*>(nullptr), uint32_t(n), 0, 64, s),
            "sort size");
    const size_t keyBytes = (n * sizeof(uint64_t) + 255) / 256 * 256;
    const size_t orderBytes = (n * sizeof(uint32_t) + 255) / 256 * 256;
    TG_CUDA(d->slots[kRecordSort].reserve(2 * keyBytes + 2 * orderBytes + sortBytes),
            "allocation");
    char* sortBase = static_cast<char*>(d->slots[kRecordSort].ptr);
    uint64_t* keys[2] = {reinterpret_cast<uint64_t*>(sortBase),
                         reinterpret_cast<uint64_t*>(sortBase + keyBytes)};
    uint32_t* order[2] = {reinterpret_cast<uint32_t*>(sortBase + 2 * keyBytes),
                          reinterpret_cast<uint32_t*>(sortBase + 2 * keyBytes + orderBytes)};
    void* sortTemp = sortBase + 2 * keyBytes + 2 * orderBytes;
    int cur = 0;  // order[cur] holds the order so far
    for (int field = 0; field < 3; ++field) {
        order_keys_kernel<<<blocks, 256, 0, s>>>(dCraters, uint32_t(n),
                                                 field == 0 ? nullptr : order[cur], field, keys[0],
                                                 order[cur]);
        TG_CUDA(cudaGetLastError(), "order keys launch");
        size_t bytes = sortBytes;
        TG_CUDA(cub::DeviceRadixSort::SortPairs(sortTemp, bytes, keys[0], keys[1], order[cur],
                                                order[cur ^ 1], uint32_t(n), 0, 64, s),
                "sort");
        cur ^= 1;
    }
    const uint32_t* applyOrder = order[cur];
    record_count_kernel<<<blocks, 256, 0, s>>>(dCraters, applyOrder, uint32_t(n), k, recordAt,
                                               dataAt);
    TG_CUDA(cudaGetLastError(), "record count launch");
    uint32_t* scratch = static_cast<uint32_t*>(d->slots[kScan].ptr);
    TG_CUDA(launch_exclusive_scan(recordAt, uint32_t(n), scratch, s), "scan launch");
    TG_CUDA(launch_exclusive_scan(dataAt, uint32_t(n), scratch, s), "scan launch");
    if (!query) {
        record_write_kernel<<<blocks, 256, 0, s>>>(
            dCraters, applyOrder, uint32_t(n), k, dExtras, recordAt, dataAt,
            records ? record_capacity : 0, data ? data_capacity : 0,
            static_cast<CraterRecord*>(records), data, footprints);
        TG_CUDA(cudaGetLastError(), "record write launch");
    }
    // The totals (the scans' last words) back to the host: the one synchronization.
    uint32_t* totals = static_cast<uint32_t*>(d->recordStage);
    TG_CUDA(cudaMemcpyAsync(totals, recordAt + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy");
    TG_CUDA(cudaMemcpyAsync(totals + 1, dataAt + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    const size_t nRecords = totals[0], nFloats = totals[1];
    *n_records = nRecords;
    *n_data = std::max<size_t>(nFloats, 1);
    if (nFloats == 0 && data != nullptr && data_capacity >= 1) {
        // An empty batch still hands the kernel one data float, 0.
        TG_CUDA(cudaMemsetAsync(data, 0, sizeof(float), s), "clear");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    }
    if ((records != nullptr || footprints != nullptr) && record_capacity < nRecords) {
        return fail(TG_ERROR_ARGUMENT, "record capacity %zu below the batch's %zu records",
                    record_capacity, nRecords);
    }
    if (data != nullptr && data_capacity < *n_data) {
        return fail(TG_ERROR_ARGUMENT, "data capacity %zu below the batch's %zu floats",
                    data_capacity, *n_data);
    }
    return TG_OK;
}

}  // extern "C"
