// The batched form: many tiles of different sizes, spacings and places evaluated together.
//
// Binning (launch_batch_bin), once per batch over all its tiles:
//   count   - one warp per crater record (thread per boulder): its footprint window on its own
//             tile's grid (the reference's CratersOnRaster / ReliefBox windows, as the plain
//             path computes them) and one count per bin of that tile it covers;
//   scan    - one exclusive prefix sum over the bins of every tile;
//   scatter - the 160-byte BinEntry (64-byte BoulderEntry) into each covered bin.
// Evaluation (launch_batch_evaluate) is ONE persistent launch: each CTA takes the next bin from
// a device work-queue cursor, finds its tile, and for the bin's cells
//   1. evaluates the source fBm with world-to-lattice offsets split in double per tile and octave
//      (OctaveAnchor), so cells millions of meters from the origin keep their lattice fraction
//      to float precision;
//   2. adds the bin's craters (entries staged in shared memory by TMA bulk copies, warp-ballot
//      culling, FP64 accumulation of FP32 contributions, as the plain path);
//   3. max-composites the bin's boulders (FP64 dome relief, as the plain path);
//   4. writes each cell once.
// The launches read their sizes from the BatchHeader in device memory, so one captured CUDA
// graph serves every batch that fits the plan's capacities.
//
// Built with -fmad=false: every fused multiply-add is written out, so heights are the same bits
// whichever kernel shape (bin size, cells per thread) the autotuner picks.
#include <utility>

#include "binning.cuh"
#include "crater_math.cuh"
#include "ds_tile.cuh"
#include "kernels.h"
#include "noise_math.cuh"

namespace tgb {
namespace {

using namespace binning;

constexpr uint32_t kStageBytes = 15360;  // one staging buffer: 96 crater or 240 boulder entries
constexpr uint32_t kCraterChunk = kStageBytes / sizeof(BinEntry);
constexpr uint32_t kBoulderChunk = kStageBytes / sizeof(BoulderEntry);
static_assert(kCraterChunk * sizeof(BinEntry) == kStageBytes, "whole crater entries per stage");
static_assert(kBoulderChunk * sizeof(BoulderEntry) == kStageBytes, "whole boulder entries");

constexpr uint32_t kLcgA = 1664525u, kLcgC = 1013904223u;

// Perlin's quintic fade and the lerp (include/terraingen/noise/lattice.h:76-86) with explicit
// fused multiply-adds. This unit is built with -fmad=false, so these are the only contractions:
// a cell's height does not depend on how a kernel shape happens to be compiled.
__device__ __forceinline__ float fade_fma(float t) {
    return t * t * t * fmaf(t, fmaf(t, 6.0f, -15.0f), 10.0f);
}

__device__ __forceinline__ float lerp_fma(float t, float a, float b) {
    return fmaf(t, b - a, a);
}

// pcg3d's x word for a corner whose first LCG step is already applied (hash.h:40-57).
__device__ __forceinline__ uint32_t corner_hash(uint32_t x, uint32_t y, uint32_t z) {
    x += y * z;
    y += z * x;
    z += x * y;
    x ^= x >> 16u;
    y ^= y >> 16u;
    z ^= z >> 16u;
    return x + y * z;
}

// --- binning -------------------------------------------------------------------------------

// The ref holding pair `p` of a prefix numbering: the last ref whose first pair is at or before
// p (refs with no pairs share their successor's first pair and are passed over).
template <typename First>
__device__ __forceinline__ uint32_t ref_of_pair(const BatchRef* refs, uint32_t n, uint32_t p,
                                                First first) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first(refs[mid]) <= p) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

__device__ __forceinline__ bool is_points(const BatchTile& t) {
    return t.kind == kTilePoints;
}

// A (ref, record) pair's place: its record, data base, item, and footprint (grid tiles: the
// reference-tile box; point sets: the disk).
struct PairSpot {
    uint32_t record, dataBase, tile;
    int4 box;         // empty: x > y
    double x, y, reach;
};

__device__ __forceinline__ PairSpot pair_spot(const BatchView& v, uint32_t p, uint32_t nrefs) {
    const BatchRef ref =
        v.refs[ref_of_pair(v.refs, nrefs, p, [](const BatchRef& r) { return r.recordPairs; })];
    PairSpot s;
    s.record = ref.recordBegin + (p - ref.recordPairs);
    s.dataBase = ref.dataBase;
    s.tile = ref.tile;
    return s;
}

// Counts of the bins each (ref, record) pair covers. The lanes of a warp take 32 pairs (each lane
// one footprint: CratersOnRaster's window on a grid tile, as the plain path, or the disk a point
// set's blocks are tested against); then the warp spreads each pair's bins over its lanes.
__global__ void batch_crater_count_kernel(const CraterShapeKernel k, const BatchView v,
                                          uint32_t tpbX, uint32_t tpbY) {
    const uint32_t n = v.header->refRecords, nrefs = v.header->refs;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t first = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; first < n;
         first += warps * 32u) {
        const uint32_t p = first + lane;
        PairSpot me{0, 0, 0, make_int4(1, 0, 1, 0), 0.0, 0.0, 0.0};
        if (p < n) {
            me = pair_spot(v, p, nrefs);
            me.box = make_int4(1, 0, 1, 0);
            const BatchTile& t = v.tiles[me.tile];
            const CraterRecord r = v.records[me.record];
            const float* data = v.data + me.dataBase;
            float cull = 0.0f;
            if (t.kind == kTileIndexedPoints) {
                // Read from the resident cell lists, not binned.
            } else if (is_points(t)) {
                const CraterReach c = crater_reach(k, r, data, v.footprints, me.record);
                me.x = c.x;
                me.y = c.y;
                me.reach = c.reach;
                cull = c.cull;
                me.box = make_int4(0, 0, 0, 0);  // non-empty: the blocks are tested below
            } else {
                const Footprint f = crater_footprint(k, r, data, v.footprints, me.record, t.grid);
                me.box = f.tiles;
                cull = f.cull;
            }
            if (me.box.x <= me.box.y) {
                if (r.hasDatum == 1u) {
                    atomicOr(&v.header->flags, 1u);
                }
                if (crater_heavy(r)) {
                    atomicOr(&v.header->flags, 8u);
                }
            }
            v.craterBoxes[p] = me.box;
            v.craterCulls[p] = cull;
        }
        const uint32_t live = __ballot_sync(0xffffffffu, me.box.x <= me.box.y);
        for (uint32_t rest = live; rest != 0u; rest &= rest - 1u) {
            const int q = __ffs(rest) - 1;
            const int4 box = make_int4(__shfl_sync(0xffffffffu, me.box.x, q),
                                       __shfl_sync(0xffffffffu, me.box.y, q),
                                       __shfl_sync(0xffffffffu, me.box.z, q),
                                       __shfl_sync(0xffffffffu, me.box.w, q));
            const uint32_t tile = __shfl_sync(0xffffffffu, me.tile, q);
            const BatchTile& t = v.tiles[tile];
            if (is_points(t)) {
                const double x = __shfl_sync(0xffffffffu, me.x, q);
                const double y = __shfl_sync(0xffffffffu, me.y, q);
                const double reach = __shfl_sync(0xffffffffu, me.reach, q);
                for (uint32_t b = lane; b < t.binsX; b += 32u) {
                    if (disk_meets_box(x, y, reach, v.pointBoxes + 4 * size_t(t.binBase + b))) {
                        atomicAdd(v.craterCounts + t.binBase + b, 1u);
                    }
                }
                continue;
            }
            const uint32_t bx0 = uint32_t(box.x) / tpbX, bx1 = uint32_t(box.y) / tpbX;
            const uint32_t by0 = uint32_t(box.z) / tpbY, by1 = uint32_t(box.w) / tpbY;
            const uint32_t wide = bx1 - bx0 + 1u;
            const uint32_t total = wide * (by1 - by0 + 1u);
            for (uint32_t c = lane; c < total; c += 32u) {
                atomicAdd(v.craterCounts + t.binBase + (by0 + c / wide) * t.binsX + bx0 + c % wide,
                          1u);
            }
        }
    }
}

// The 160-byte BinEntry of each pair into every bin it covers: the lanes of a warp read 32 pairs'
// boxes, then the warp spreads each pair's bins over its lanes. The entry's index field holds the
// pair's data base, where the shaping reads the record's data.
__global__ void batch_crater_scatter_kernel(const CraterShapeKernel k, const BatchView v,
                                            uint32_t tpbX, uint32_t tpbY) {
    const uint32_t n = v.header->refRecords, nrefs = v.header->refs;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t first = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; first < n;
         first += warps * 32u) {
        const uint32_t p = first + lane;
        PairSpot me{0, 0, 0, make_int4(1, 0, 1, 0), 0.0, 0.0, 0.0};
        float cull = 0.0f;
        if (p < n) {
            me.box = v.craterBoxes[p];
            if (me.box.x <= me.box.y) {
                const int4 box = me.box;
                me = pair_spot(v, p, nrefs);
                me.box = box;
                cull = v.craterCulls[p];
                if (is_points(v.tiles[me.tile])) {
                    const CraterReach c = crater_reach(k, v.records[me.record],
                                                       v.data + me.dataBase, v.footprints,
                                                       me.record);
                    me.x = c.x;
                    me.y = c.y;
                    me.reach = c.reach;
                }
            }
        }
        const uint32_t live = __ballot_sync(0xffffffffu, me.box.x <= me.box.y);
        for (uint32_t rest = live; rest != 0u; rest &= rest - 1u) {
            const int q = __ffs(rest) - 1;
            const int4 box = make_int4(__shfl_sync(0xffffffffu, me.box.x, q),
                                       __shfl_sync(0xffffffffu, me.box.y, q),
                                       __shfl_sync(0xffffffffu, me.box.z, q),
                                       __shfl_sync(0xffffffffu, me.box.w, q));
            const uint32_t tile = __shfl_sync(0xffffffffu, me.tile, q);
            const uint32_t record = __shfl_sync(0xffffffffu, me.record, q);
            int4 tail;
            tail.x = int(uint32_t(box.x) | (uint32_t(box.y) << 16));
            tail.y = int(uint32_t(box.z) | (uint32_t(box.w) << 16));
            tail.z = __float_as_int(__shfl_sync(0xffffffffu, cull, q));
            tail.w = int(__shfl_sync(0xffffffffu, me.dataBase, q));
            const int4* src = reinterpret_cast<const int4*>(v.records + record);
            auto put = [&](uint32_t b) {
                const uint32_t slot = v.craterCounts[b] + atomicAdd(v.craterCursor + b, 1u);
                if (slot >= v.craterCapacity) {
                    return;  // counted in the header's entry total; the host re-plans
                }
                int4* dst = reinterpret_cast<int4*>(v.craterEntries + slot);
#pragma unroll
                for (int w = 0; w < 9; ++w) {
                    dst[w] = __ldg(src + w);
                }
                dst[9] = tail;
            };
            const BatchTile& t = v.tiles[tile];
            if (is_points(t)) {
                const double x = __shfl_sync(0xffffffffu, me.x, q);
                const double y = __shfl_sync(0xffffffffu, me.y, q);
                const double reach = __shfl_sync(0xffffffffu, me.reach, q);
                for (uint32_t b = lane; b < t.binsX; b += 32u) {
                    if (disk_meets_box(x, y, reach, v.pointBoxes + 4 * size_t(t.binBase + b))) {
                        put(t.binBase + b);
                    }
                }
                continue;
            }
            const uint32_t bx0 = uint32_t(box.x) / tpbX, bx1 = uint32_t(box.y) / tpbX;
            const uint32_t by0 = uint32_t(box.z) / tpbY, by1 = uint32_t(box.w) / tpbY;
            const uint32_t wide = bx1 - bx0 + 1u;
            const uint32_t total = wide * (by1 - by0 + 1u);
            for (uint32_t c = lane; c < total; c += 32u) {
                put(t.binBase + (by0 + c / wide) * t.binsX + bx0 + c % wide);
            }
        }
    }
}

// The lean path's (amplitude cos phase, amplitude sin phase) at each record's data offsets. A
// record named by several refs is written with the same values by each.
__global__ void batch_harmonics_kernel(const BatchView v) {
    const uint32_t n = v.header->refRecords, nrefs = v.header->refs;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const BatchRef ref =
            v.refs[ref_of_pair(v.refs, nrefs, p, [](const BatchRef& r) { return r.recordPairs; })];
        const uint32_t i = ref.recordBegin + (p - ref.recordPairs);
        const uint32_t offset = ref.dataBase + v.records[i].harmonicOffset;
        const uint32_t count = v.records[i].harmonicCount;
        for (uint32_t h = 0; h < count; ++h) {
            const float amplitude = __ldg(v.data + offset + 2u * h);
            const float phase = __ldg(v.data + offset + 2u * h + 1u);
            float s, c;
            sincosf(phase, &s, &c);
            v.harmonics[offset + 2u * h] = amplitude * c;
            v.harmonics[offset + 2u * h + 1u] = amplitude * s;
        }
    }
}

// One thread per (ref, boulder) pair: the bins its box's pixel window covers (point sets: the
// blocks its box meets).
__global__ void batch_boulder_count_kernel(const BatchView v, uint32_t binW, uint32_t binH) {
    const uint32_t n = v.header->refBoulders, nrefs = v.header->refs;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const BatchRef ref =
            v.refs[ref_of_pair(v.refs, nrefs, p, [](const BatchRef& r) { return r.boulderPairs; })];
        const uint32_t i = ref.boulderBegin + (p - ref.boulderPairs);
        const BatchTile& t = v.tiles[ref.tile];
        const BoulderRecord b = v.boulders[i];
        // ReliefBox on a plane (boulder_relief.cpp:24): reach 0.5 (diameter + width).
        const double reach = 0.5 * (b.diameter + t.boulderWidth);
        int4 w = make_int4(1, 0, 1, 0);
        if (b.weight > 0.0) {
            if (is_points(t)) {
                w = make_int4(INT32_MIN, INT32_MAX, INT32_MIN, INT32_MAX);
                for (uint32_t q = 0; q < t.binsX; ++q) {
                    const double* box = v.pointBoxes + 4 * size_t(t.binBase + q);
                    if (b.x + reach >= box[0] && b.x - reach <= box[2] && b.y + reach >= box[1] &&
                        b.y - reach <= box[3]) {
                        atomicAdd(v.boulderCounts + t.binBase + q, 1u);
                    }
                }
            } else {
                int c0, c1, r0, r1;
                window_of(t.grid, b.x - reach, b.y - reach, b.x + reach, b.y + reach, c0, c1, r0,
                          r1);
                if (c0 < c1 && r0 < r1) {
                    w = make_int4(c0, c1, r0, r1);
                    const uint32_t bx0 = uint32_t(c0) / binW, bx1 = uint32_t(c1 - 1) / binW;
                    const uint32_t by0 = uint32_t(r0) / binH, by1 = uint32_t(r1 - 1) / binH;
                    for (uint32_t by = by0; by <= by1; ++by) {
                        for (uint32_t bx = bx0; bx <= bx1; ++bx) {
                            atomicAdd(v.boulderCounts + t.binBase + by * t.binsX + bx, 1u);
                        }
                    }
                }
            }
        }
        v.boulderWindows[p] = w;
    }
}

__global__ void batch_boulder_scatter_kernel(const BatchView v, uint32_t binW, uint32_t binH) {
    const uint32_t n = v.header->refBoulders, nrefs = v.header->refs;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int4 w = v.boulderWindows[p];
        if (w.x >= w.y) {
            continue;
        }
        const BatchRef ref =
            v.refs[ref_of_pair(v.refs, nrefs, p, [](const BatchRef& r) { return r.boulderPairs; })];
        const uint32_t i = ref.boulderBegin + (p - ref.boulderPairs);
        const BatchTile& t = v.tiles[ref.tile];
        const BoulderRecord b = v.boulders[i];
        BoulderEntry e;
        e.x = b.x;
        e.y = b.y;
        e.radius = 0.5 * b.diameter;
        e.exposed = b.exposedHeight;
        e.weight = b.weight;
        e.c0 = w.x;
        e.c1 = w.y;
        e.r0 = w.z;
        e.r1 = w.w;
        e.pad_ = 0.0;
        auto put = [&](uint32_t bin) {
            const uint32_t slot = v.boulderCounts[bin] + atomicAdd(v.boulderCursor + bin, 1u);
            if (slot < v.boulderCapacity) {
                v.boulderEntries[slot] = e;
            }
        };
        if (is_points(t)) {
            const double reach = 0.5 * (b.diameter + t.boulderWidth);
            for (uint32_t q = 0; q < t.binsX; ++q) {
                const double* box = v.pointBoxes + 4 * size_t(t.binBase + q);
                if (b.x + reach >= box[0] && b.x - reach <= box[2] && b.y + reach >= box[1] &&
                    b.y - reach <= box[3]) {
                    put(t.binBase + q);
                }
            }
            continue;
        }
        const uint32_t bx0 = uint32_t(w.x) / binW, bx1 = uint32_t(w.y - 1) / binW;
        const uint32_t by0 = uint32_t(w.z) / binH, by1 = uint32_t(w.w - 1) / binH;
        for (uint32_t by = by0; by <= by1; ++by) {
            for (uint32_t bx = bx0; bx <= bx1; ++bx) {
                put(t.binBase + by * t.binsX + bx);
            }
        }
    }
}

// The entry totals the scans left after the last bin, for the host's capacity check.
__global__ void batch_totals_kernel(const BatchView v) {
    v.header->craterEntries = v.craterCounts[v.capacityBins];
    v.header->boulderEntries = v.boulderCounts[v.capacityBins];
}

// --- the persistent evaluation -------------------------------------------------------------

// Issues the bulk copy of chunk `c` of `count` entries (of `entryBytes`) from `src` into stage
// buffer c & 1. Thread 0 only.
__device__ __forceinline__ void issue_chunk(unsigned char (*stage)[kStageBytes], uint64_t* bars,
                                            const unsigned char* src, uint32_t entryBytes,
                                            uint32_t chunk, uint32_t count, uint32_t c) {
    const uint32_t s = c & 1u;
    const uint32_t n = min(chunk, count - c * chunk);
    const uint32_t bytes = n * entryBytes;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bars[s], bytes);
    bulk_copy_g2s(&stage[s][0], src + size_t(c) * chunk * entryBytes, bytes, &bars[s]);
}

// Perlin noise at one lattice point split into cell (ix, iy) and fraction (fx, fy), its four
// corner hashes given (PerlinNoise2, include/terraingen/noise/perlin.h:72-98).
__device__ __forceinline__ float perlin_at(uint32_t h00, uint32_t h10, uint32_t h01, uint32_t h11,
                                          float fx, float fy) {
    const float n00 = noise::gradient2(h00, fx, fy);
    const float n10 = noise::gradient2(h10, fx - 1.0f, fy);
    const float n01 = noise::gradient2(h01, fx, fy - 1.0f);
    const float n11 = noise::gradient2(h11, fx - 1.0f, fy - 1.0f);
    const float u = fade_fma(fx), vv = fade_fma(fy);
    return 1.41421356237309505f * lerp_fma(vv, lerp_fma(u, n00, n10), lerp_fma(u, n01, n11));
}

// sum + err += w * n, keeping the product's and the sum's rounding errors in err.
__device__ __forceinline__ void accumulate(float& sum, float& err, float w, float n) {
    const float t = w * n;
    const float te = fmaf(w, n, -t);  // w * n - t, exactly
    const float s = sum + t;
    const float bp = s - sum;
    const float se = (sum - (s - bp)) + (t - bp);  // TwoSum: sum + t - s, exactly
    sum = s;
    err += se + te;
}

__device__ __forceinline__ void corners(int32_t ix, int32_t iy, uint32_t sz, uint32_t& h00,
                                        uint32_t& h10, uint32_t& h01, uint32_t& h11) {
    const uint32_t ax0 = uint32_t(ix) * kLcgA + kLcgC, ax1 = ax0 + kLcgA;
    const uint32_t ay0 = uint32_t(iy) * kLcgA + kLcgC, ay1 = ay0 + kLcgA;
    h00 = corner_hash(ax0, ay0, sz);
    h10 = corner_hash(ax1, ay0, sz);
    h01 = corner_hash(ax0, ay1, sz);
    h11 = corner_hash(ax1, ay1, sz);
}

// The source at a point: Fractal2's octaves with each lattice position split in double, summed
// with compensation (see the grid path), as elevation + amplitude * sum / total.
__device__ __forceinline__ float point_source(const BatchNoise& noise, double x, double y) {
    float sum = 0.0f, err = 0.0f;
    for (int o = 0; o < noise.octaves; ++o) {
        const double px = fma(fma(x, noise.tc[o], -y * noise.ts[o]), noise.frequency[o],
                              noise.ox[o]);
        const double py = fma(fma(x, noise.ts[o], y * noise.tc[o]), noise.frequency[o],
                              noise.oy[o]);
        const double lx = floor(px), ly = floor(py);
        uint32_t h00, h10, h01, h11;
        corners(int32_t(uint32_t(uint64_t(int64_t(lx)))), int32_t(uint32_t(uint64_t(int64_t(ly)))),
                noise.seedTerm[o], h00, h10, h01, h11);
        accumulate(sum, err, noise.weight[o],
                   perlin_at(h00, h10, h01, h11, float(px - lx), float(py - ly)));
    }
    return float(fma(noise.scale, double(sum) + double(err), double(noise.elevation)));
}

// Level-0 diamond-square nodes from the batch's source: node (col, row) is the post at
// (col, row) * spacing, the fBm there as point_source evaluates it (rounded to float, as a DEM's
// posts are).
struct PostsFromSource {
    const BatchNoise& noise;
    double spacing;
    __device__ __forceinline__ double operator()(int64_t col, int64_t row) const {
        return double(point_source(noise, double(col) * spacing, double(row) * spacing));
    }
};

// The diamond-square pass of a batch: persistent CTAs take the jobs' blocks in turn (a block's
// job by binary search over the jobs' first blocks) and write each block's base heights into the
// batch's output.
template <bool kSpline>
__global__ void __launch_bounds__(kDsTileThreads, 3) batch_ds_kernel(const BatchNoise noise,
                                                                 const BatchView v) {
    extern __shared__ double pool[];
    __shared__ DsShared sh;
    __shared__ uint32_t sJob;
    const BatchHeader* header = v.header;
    const uint32_t jobs = header->dsJobs, blocks = header->dsBlocks;
    float* const heights = header->heights;
    for (uint32_t g = blockIdx.x; g < blocks; g += gridDim.x) {
        if (threadIdx.x == 0) {
            uint32_t lo = 0, hi = jobs;
            while (hi - lo > 1u) {
                const uint32_t mid = (lo + hi) >> 1;
                if (v.dsFirst[mid] <= g) {
                    lo = mid;
                } else {
                    hi = mid;
                }
            }
            sJob = lo;
        }
        __syncthreads();
        const DsTile& t = v.dsJobs[sJob];
        const PostsFromSource posts{noise, t.postSpacing};
        ds_block<kSpline>(t, g - v.dsFirst[sJob], posts, heights + t.heightOffset, pool, sh);
        __syncthreads();  // the next block's boxes overwrite this one's shared state
    }
}

// The points' diamond-square pass: each warp takes one point at a time (its node boxes are a
// few nodes wide), eight warps a CTA, each with its own node buffers.
template <bool kSpline>
__global__ void __launch_bounds__(256, 3) batch_ds_points_kernel(const BatchNoise noise,
                                                              const BatchView v) {
    extern __shared__ double pointPool[];
    __shared__ DsShared sh[8];
    const uint32_t warp = threadIdx.x >> 5u;
    const BatchHeader* header = v.header;
    const uint32_t jobs = header->dsPointJobs, points = header->dsPoints;
    float* const heights = header->heights;
    for (uint32_t g = blockIdx.x * 8u + warp; g < points; g += gridDim.x * 8u) {
        uint32_t lo = 0, hi = jobs;
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (v.dsPointFirst[mid] <= g) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const DsTile& t = v.dsPointJobs[lo];
        const PostsFromSource posts{noise, t.postSpacing};
        ds_block<kSpline>(t, g - v.dsPointFirst[lo], posts, heights + t.heightOffset,
                          pointPool + size_t(warp) * kDsPointPool, sh[warp], WarpGroup());
        __syncwarp();  // the next point's boxes overwrite this one's shared state
    }
}

// One point of an indexed point set per thread: the source, then the craters of its resident
// region's cell list (each within its cull distance), one write. Threads run independently.
template <bool kFast>
__device__ __forceinline__ void indexed_points(const CraterShapeKernel& k,
                                               const crater::FastKernel& fk,
                                               const BatchNoise& noise, const BatchView& v,
                                               const BatchTile& t, uint32_t i, float* heights,
                                               uint32_t& pairs) {
    if (i >= t.grid.width) {
        return;
    }
    const size_t at = size_t(t.pointBase) + i;
    const double x = v.points[2 * at], y = v.points[2 * at + 1];
    const float base =
        noise.baseInOutput ? heights[t.heightOffset + i] : point_source(noise, x, y);
    double acc = double(base);
    // The point's region from the set's region table.
    const double side = t.grid.pixelWidth;
    const uint32_t tw = t.grid.height, th = t.pitch;
    const int rx = min(max(int(floor((x - t.grid.originX) / side)), 0), int(tw) - 1);
    const int ry = min(max(int(floor((y - t.grid.originY) / side)), 0), int(th) - 1);
    const uint32_t region = v.pointTable[t.tableBase + uint32_t(ry) * tw + uint32_t(rx)];
    if (region == 0xffffffffu) {
        heights[t.heightOffset + i] = base;  // no region: the source alone (not reached)
        return;
    }
    const PointRegion pr = v.pointRegions[region];
    const int gx = min(max(int(floor((x - pr.x0) / pr.cell)), 0), int(pr.g) - 1);
    const int gy = min(max(int(floor((y - pr.y0) / pr.cell)), 0), int(pr.g) - 1);
    const uint32_t* lists = v.pointLists + pr.listBase;
    const uint32_t cell = uint32_t(gy) * pr.g + uint32_t(gx);
    const uint32_t* entries = lists + pr.g * pr.g + 1;
    const float pxh = float(x), pxl = float(x - double(pxh));
    const float pyh = float(y), pyl = float(y - double(pyh));
    const float* data = v.data + pr.dataBase;
    const float* harmonics = v.harmonics + pr.dataBase;
    for (uint32_t e = lists[cell]; e < lists[cell + 1]; ++e) {
        const uint32_t rec = pr.recBase + entries[e];
        const CraterRecord r = v.records[rec];
        const float cull = v.culls[rec];
        const float dx = crater::split_difference(pxh, pxl, r.x, r.xLow);
        const float dy = crater::split_difference(pyh, pyl, r.y, r.yLow);
        if (!(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) < cull * cull)) {
            continue;
        }
        ++pairs;
        if (kFast) {
            bool reached;
            const float shaped = crater::fast_contribution(fk, harmonics, r, dx, dy, reached);
            if (reached) {
                acc += double(shaped);
            }
        } else {
            const crater::Contribution q = crater::crater_contribution(k, data, r, dx, dy);
            if (q.reached) {
                acc += double(q.shaped);
            }
        }
    }
    heights[t.heightOffset + i] = float(acc);
}

template <int kBinW, int kBinH, int kCells, bool kFast>
__global__ void __launch_bounds__(kBinW* kBinH / kCells, 768 / (kBinW * kBinH / kCells))
    batch_evaluate_kernel(const CraterShapeKernel k, const BatchNoise noise, const BatchView v) {
    constexpr uint32_t kRowThreads = kBinW / kCells;  // threads along one row of a bin
    constexpr uint32_t kBinCellCount = kBinW * kBinH;  // cells of a bin, points of a point block
    static_assert(kBinW % kCells == 0 && kRefTileCells % kCells == 0, "cells per thread");
    static_assert(kBinW % kRefTileCells == 0 && kBinH % kRefTileCells == 0, "bins of 16-tiles");

    __shared__ __align__(128) unsigned char stage[2][kStageBytes];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t sItem, sTile;
    // Dynamic: per warp, FP64 accumulators of its cells and the queue of (crater, cell) pairs.
    constexpr uint32_t kWarpCells = 32u * kCells;
    constexpr uint32_t kQueueCap = 31u + kWarpCells;
    extern __shared__ double craterAcc[];
    uint16_t* const craterQueue =
        reinterpret_cast<uint16_t*>(craterAcc + (kBinW * kBinH / kCells / 32) * kWarpCells);

    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const crater::FastKernel fk{k.profile.simple, k.profile.rim, k.reachRadii};
    BatchHeader* header = v.header;
    const uint32_t nbins = min(header->bins, header->evalEnd), ntiles = header->tiles;
    float* const heights = header->heights;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    uint32_t phase[2] = {0u, 0u};
    uint32_t craterPairs = 0, boulderPairs = 0;

    for (;;) {
        __syncthreads();  // the previous bin's stage and item are no longer read
        if (tid == 0) {
            const uint32_t item = atomicAdd(&header->next, 1u);
            uint32_t lo = 0;
            if (item < nbins) {
                // The last tile whose first bin is at or before the item.
                uint32_t hi = ntiles;
                while (hi - lo > 1u) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (v.tiles[mid].binBase <= item) {
                        lo = mid;
                    } else {
                        hi = mid;
                    }
                }
            }
            sItem = item;
            sTile = lo;
        }
        __syncthreads();
        const uint32_t item = sItem;
        if (item >= nbins) {
            break;
        }
        const BatchTile& t = v.tiles[sTile];
        const Grid grid = t.grid;
        const uint32_t local = item - t.binBase;
        if (t.kind == kTileIndexedPoints) {
            indexed_points<kFast>(k, fk, noise, v, t, local * (kBinW * kBinH / kCells) + tid,
                                  heights, craterPairs);
            continue;
        }
        const bool points = t.kind == kTilePoints;
        // Grid: this thread's kCells cells of one row. Point set: kCells consecutive points.
        uint32_t row = 0, col0 = 0, first = 0;
        bool live[kCells];
        if (points) {
            first = local * kBinCellCount + tid * kCells;
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                live[j] = first + j < grid.width;
            }
        } else {
            const uint32_t binX = local % t.binsX, binY = local / t.binsX;
            row = binY * kBinH + tid / kRowThreads;
            col0 = binX * kBinW + (tid % kRowThreads) * kCells;
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                live[j] = row < grid.height && col0 + j < grid.width;
            }
        }
        // Cell centers (Raster::CellCenter) or points, in double.
        double xd[kCells], yd[kCells];
#pragma unroll
        for (int j = 0; j < kCells; ++j) {
            if (points) {
                const uint32_t i = live[j] ? first + j : 0u;
                xd[j] = v.points[2 * (size_t(t.pointBase) + i)];
                yd[j] = v.points[2 * (size_t(t.pointBase) + i) + 1];
            } else {
                xd[j] = grid.originX + (double(col0 + j) + 0.5) * grid.pixelWidth +
                        (double(row) + 0.5) * grid.rowRotation;
                yd[j] = grid.originY + (double(col0 + j) + 0.5) * grid.colRotation +
                        (double(row) + 0.5) * grid.pixelHeight;
            }
        }

        // 1. The source: the base a diamond-square pass already wrote into the output, or
        //    Fractal2's octaves.
        float h[kCells];
        if (noise.baseInOutput) {
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                h[j] = 0.0f;
                if (live[j]) {
                    h[j] = points ? heights[t.heightOffset + v.pointIndex[t.pointBase + first + j]]
                                  : heights[t.heightOffset + size_t(row) * t.pitch + col0 + j];
                }
            }
        } else {
            // Fractal2's octaves (fractal.h:219-240). Grid cells take their lattice
            //    position from the tile's per-octave anchor (split in double) plus float steps;
            //    points split their own position in double. Corner hashes are reused while the
            //    lattice cell does not change.
            // Compensated octave sums: sum + err carries the weighted octaves to about twice float
            // precision (each product's rounding from an FMA residual, each sum's by TwoSum), so a
            // source of kilometers keeps its millimeters.
            float sum[kCells], err[kCells];
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                sum[j] = 0.0f;
                err[j] = 0.0f;
            }
            for (int o = 0; o < noise.octaves; ++o) {
                const uint32_t sz = noise.seedTerm[o];
                const float w = noise.weight[o];
                int32_t cx = INT32_MIN, cy = INT32_MIN;
                uint32_t h00 = 0, h10 = 0, h01 = 0, h11 = 0;
                if (points) {
                    const double tc = noise.tc[o], ts = noise.ts[o], f = noise.frequency[o];
#pragma unroll
                    for (int j = 0; j < kCells; ++j) {
                        const double px = fma(fma(xd[j], tc, -yd[j] * ts), f, noise.ox[o]);
                        const double py = fma(fma(xd[j], ts, yd[j] * tc), f, noise.oy[o]);
                        const double lx = floor(px), ly = floor(py);
                        const int32_t ix = int32_t(uint32_t(uint64_t(int64_t(lx))));
                        const int32_t iy = int32_t(uint32_t(uint64_t(int64_t(ly))));
                        if (ix != cx || iy != cy) {
                            cx = ix;
                            cy = iy;
                            corners(ix, iy, sz, h00, h10, h01, h11);
                        }
                        accumulate(sum[j], err[j], w,
                                   perlin_at(h00, h10, h01, h11, float(px - lx), float(py - ly)));
                    }
                } else {
                    const OctaveAnchor a = v.anchors[t.anchorBase + o];
                    // Each cell from its own column, so heights do not depend on the kernel shape.
                    const float fr = float(row);
                    const float px = fmaf(fr, a.ay, a.fx);
                    const float py = fmaf(fr, a.by, a.fy);
#pragma unroll
                    for (int j = 0; j < kCells; ++j) {
                        const float qx = fmaf(float(col0 + j), a.ax, px);
                        const float qy = fmaf(float(col0 + j), a.bx, py);
                        const float lx = floorf(qx), ly = floorf(qy);
                        const int32_t ix = int32_t(uint32_t(a.ix) + uint32_t(int32_t(lx)));
                        const int32_t iy = int32_t(uint32_t(a.iy) + uint32_t(int32_t(ly)));
                        if (ix != cx || iy != cy) {
                            cx = ix;
                            cy = iy;
                            corners(ix, iy, sz, h00, h10, h01, h11);
                        }
                        accumulate(sum[j], err[j], w, perlin_at(h00, h10, h01, h11, qx - lx, qy - ly));
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                // elevation + amplitude * sum / total, formed once per cell in double.
                h[j] = float(fma(noise.scale, double(sum[j]) + double(err[j]),
                                 double(noise.elevation)));
            }
        }

        // 2. Craters: each entry's data at its ref's base (the BinEntry's index field).
        const uint32_t cFirst = v.craterCounts[item];
        const uint32_t cEnd = min(v.craterCounts[item + 1], v.craterCapacity);
        const uint32_t cCount = cEnd > cFirst ? cEnd - cFirst : 0u;
        if (cCount > 0u) {
            // Split positions of the cell centers (MakeSplitPoint, crater_kernel.cpp:303): grid
            // rows take the row center at column 0 (the reference's strips carry one y per row),
            // points their own y. `split_of` gives any cell of this warp's, so a lane can shape
            // another lane's cell.
            const uint32_t warpBase = tid & ~31u;
            auto split_of = [&](uint32_t owner, int j, float& xh, float& xl, float& yh,
                                float& yl) {
                double x, y;
                if (points) {
                    const uint32_t f = local * kBinCellCount + (warpBase + owner) * kCells;
                    const uint32_t i = f + j < grid.width ? f + j : 0u;
                    x = v.points[2 * (size_t(t.pointBase) + i)];
                    y = v.points[2 * (size_t(t.pointBase) + i) + 1];
                } else {
                    const uint32_t o = warpBase + owner;
                    const uint32_t binX = local % t.binsX, binY = local / t.binsX;
                    const uint32_t r = binY * kBinH + o / kRowThreads;
                    const uint32_t c = binX * kBinW + (o % kRowThreads) * kCells + j;
                    y = grid.originY + 0.5 * grid.colRotation + (double(r) + 0.5) * grid.pixelHeight;
                    x = grid.originX + (double(c) + 0.5) * grid.pixelWidth +
                        0.5 * grid.rowRotation;
                }
                xh = float(x);
                xl = float(x - double(xh));
                yh = float(y);
                yl = float(y - double(yh));
            };
            float pxh[kCells], pxl[kCells], pyh[kCells], pyl[kCells];
            double* acc = craterAcc + (tid >> 5) * kWarpCells;
            uint16_t* queue = craterQueue + (tid >> 5) * kQueueCap;
            bool anyLive = false;
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                split_of(lane, j, pxh[j], pxl[j], pyh[j], pyl[j]);
                acc[lane * kCells + j] = double(h[j]);
                anyLive |= live[j];
            }
            const int tileX = int(col0 / kRefTileCells), tileY = int(row / kRefTileCells);
            const unsigned char* src =
                reinterpret_cast<const unsigned char*>(v.craterEntries + cFirst);
            const uint32_t chunks = (cCount + kCraterChunk - 1) / kCraterChunk;
            if (tid == 0) {
                issue_chunk(stage, bars, src, sizeof(BinEntry), kCraterChunk, cCount, 0);
                if (chunks > 1) {
                    issue_chunk(stage, bars, src, sizeof(BinEntry), kCraterChunk, cCount, 1);
                }
            }
            bool failed = false;
            for (uint32_t c = 0; c < chunks; ++c) {
                const uint32_t s = c & 1u;
                if (!mbar_wait(&bars[s], phase[s])) {
                    failed = true;
                }
                phase[s] ^= 1u;
                if (__syncthreads_or(failed)) {
                    if (tid == 0) {
                        atomicOr(&header->flags, 2u);
                        if (c + 1 < chunks) {
                            mbar_wait(&bars[s ^ 1u], phase[s ^ 1u]);
                        }
                    }
                    return;
                }
                const BinEntry* entries = reinterpret_cast<const BinEntry*>(&stage[s][0]);
                const uint32_t n = min(kCraterChunk, cCount - c * kCraterChunk);
                // Shapes the queued pairs [from, from + count), one per lane: each entry's data
                // at its ref's base (the BinEntry's index field).
                auto drain = [&](uint32_t from, uint32_t count) {
                    if (lane < count) {
                        const uint32_t code = queue[from + lane];
                        const BinEntry& entry = entries[code >> 8];
                        const CraterRecord& r = entry.record;
                        const uint32_t cell = code & 255u;
                        float xh, xl, yh, yl;
                        split_of(cell / kCells, int(cell % kCells), xh, xl, yh, yl);
                        const float dx = crater::split_difference(xh, xl, r.x, r.xLow);
                        const float dy = crater::split_difference(yh, yl, r.y, r.yLow);
                        if (kFast) {
                            bool reached;
                            const float shaped = crater::fast_contribution(
                                fk, v.harmonics + entry.index, r, dx, dy, reached);
                            if (reached) {
                                atomicAdd(acc + cell, double(shaped));
                            }
                        } else {
                            const crater::Contribution q =
                                crater::crater_contribution(k, v.data + entry.index, r, dx, dy);
                            if (q.reached) {
                                atomicAdd(acc + cell, double(q.shaped));
                            }
                        }
                    }
                };
                uint32_t queued = 0;  // warp-uniform
                for (uint32_t e = 0; e < n; ++e) {
                    const BinEntry& entry = entries[e];
                    const CraterRecord& r = entry.record;
                    // Grid cells: every cell of each reference tile the footprint touches.
                    const bool inTile = anyLive &&
                                        (points || (tileX >= int(entry.tileX0) &&
                                                    tileX <= int(entry.tileX1) &&
                                                    tileY >= int(entry.tileY0) &&
                                                    tileY <= int(entry.tileY1)));
                    if (!__any_sync(0xffffffffu, inTile)) {
                        continue;  // none of the warp's cells is in the crater's window
                    }
                    const float cull2 = entry.cull * entry.cull;
                    uint32_t need = 0;
#pragma unroll
                    for (int j = 0; j < kCells; ++j) {
                        const float dx = crater::split_difference(pxh[j], pxl[j], r.x, r.xLow);
                        const float dy = crater::split_difference(pyh[j], pyl[j], r.y, r.yLow);
                        if (inTile && live[j] &&
                            __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)) < cull2) {
                            need |= 1u << j;
                        }
                    }
                    if (!__any_sync(0xffffffffu, need != 0u)) {
                        continue;
                    }
                    const uint32_t mine = __popc(need);
                    uint32_t before = mine;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const uint32_t other = __shfl_up_sync(0xffffffffu, before, d);
                        if (lane >= uint32_t(d)) {
                            before += other;
                        }
                    }
                    const uint32_t total = __shfl_sync(0xffffffffu, before, 31);
                    if (total == 0u) {
                        continue;
                    }
                    uint32_t slot = queued + before - mine;
                    for (int j = 0; j < kCells; ++j) {
                        if (need & (1u << j)) {
                            queue[slot++] = uint16_t((e << 8) | (lane * kCells + j));
                        }
                    }
                    craterPairs += mine;
                    queued += total;
                    __syncwarp();
                    while (queued >= 32u) {
                        queued -= 32u;
                        drain(queued, 32u);
                        __syncwarp();
                    }
                }
                if (queued > 0u) {
                    drain(0u, queued);
                    __syncwarp();
                }
                if (c + 2 < chunks) {
                    __syncthreads();  // every warp has read the buffer before it is refilled
                    if (tid == 0) {
                        issue_chunk(stage, bars, src, sizeof(BinEntry), kCraterChunk, cCount,
                                    c + 2);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                h[j] = float(acc[lane * kCells + j]);
            }
        }

        // 3. Boulders: max(height, base + weight * dome), base being the height after craters.
        const uint32_t bFirst = v.boulderCounts[item];
        const uint32_t bEnd = min(v.boulderCounts[item + 1], v.boulderCapacity);
        const uint32_t bCount = bEnd > bFirst ? bEnd - bFirst : 0u;
        if (bCount > 0u) {
            __syncthreads();  // the crater stage is no longer read
            const double width = t.boulderWidth;
            double best[kCells];
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                best[j] = double(h[j]);
            }
            const unsigned char* src =
                reinterpret_cast<const unsigned char*>(v.boulderEntries + bFirst);
            const uint32_t chunks = (bCount + kBoulderChunk - 1) / kBoulderChunk;
            if (tid == 0) {
                issue_chunk(stage, bars, src, sizeof(BoulderEntry), kBoulderChunk, bCount, 0);
                if (chunks > 1) {
                    issue_chunk(stage, bars, src, sizeof(BoulderEntry), kBoulderChunk, bCount, 1);
                }
            }
            bool failed = false;
            for (uint32_t c = 0; c < chunks; ++c) {
                const uint32_t s = c & 1u;
                if (!mbar_wait(&bars[s], phase[s])) {
                    failed = true;
                }
                phase[s] ^= 1u;
                if (__syncthreads_or(failed)) {
                    if (tid == 0) {
                        atomicOr(&header->flags, 2u);
                        if (c + 1 < chunks) {
                            mbar_wait(&bars[s ^ 1u], phase[s ^ 1u]);
                        }
                    }
                    return;
                }
                const BoulderEntry* entries = reinterpret_cast<const BoulderEntry*>(&stage[s][0]);
                const uint32_t n = min(kBoulderChunk, bCount - c * kBoulderChunk);
                for (uint32_t e = 0; e < n; ++e) {
                    const BoulderEntry& b = entries[e];
                    // Grid cells: the pixel window of the boulder's box (ForEachFeatureCell);
                    // points: wherever the dome reaches.
                    bool in[kCells];
                    bool any = false;
#pragma unroll
                    for (int j = 0; j < kCells; ++j) {
                        in[j] = live[j] &&
                                (points || (int(row) >= b.r0 && int(row) < b.r1 &&
                                            int(col0) + j >= b.c0 && int(col0) + j < b.c1));
                        any |= in[j];
                    }
                    if (!__any_sync(0xffffffffu, any)) {
                        continue;
                    }
#pragma unroll
                    for (int j = 0; j < kCells; ++j) {
                        if (in[j]) {
                            ++boulderPairs;
                            const double relief =
                                fmax(dome(b, hypot(xd[j] - b.x, yd[j] - b.y), width), 0.0);
                            if (relief > 0.0) {
                                best[j] = fmax(best[j], fma(b.weight, relief, double(h[j])));
                            }
                        }
                    }
                }
                if (c + 2 < chunks) {
                    __syncthreads();
                    if (tid == 0) {
                        issue_chunk(stage, bars, src, sizeof(BoulderEntry), kBoulderChunk, bCount,
                                    c + 2);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                h[j] = float(best[j]);
            }
        }

        // 4. One write per cell; a point to its caller's index.
        if (points) {
#pragma unroll
            for (int j = 0; j < kCells; ++j) {
                if (live[j]) {
                    heights[t.heightOffset + v.pointIndex[t.pointBase + first + j]] = h[j];
                }
            }
            continue;
        }
        float* dst = heights + t.heightOffset + size_t(row) * t.pitch + col0;
        bool all = true, none = true;
#pragma unroll
        for (int j = 0; j < kCells; ++j) {
            all &= live[j];
            none &= !live[j];
        }
        if (!none) {
            const uintptr_t address = reinterpret_cast<uintptr_t>(dst);
            if (kCells % 4 == 0 && all && (address & 15u) == 0u) {
#pragma unroll
                for (int j = 0; j < kCells; j += 4) {
                    *reinterpret_cast<float4*>(dst + j) =
                        make_float4(h[j], h[j + 1], h[j + 2], h[j + 3]);
                }
            } else if (kCells == 2 && all && (address & 7u) == 0u) {
                *reinterpret_cast<float2*>(dst) = make_float2(h[0], h[kCells - 1]);
            } else {
#pragma unroll
                for (int j = 0; j < kCells; ++j) {
                    if (live[j]) {
                        dst[j] = h[j];
                    }
                }
            }
        }
    }
    const uint32_t warpCraters = __reduce_add_sync(0xffffffffu, craterPairs);
    const uint32_t warpBoulders = __reduce_add_sync(0xffffffffu, boulderPairs);
    if (lane == 0) {
        if (warpCraters > 0) {
            atomicAdd(&header->craterPairs, (unsigned long long)warpCraters);
        }
        if (warpBoulders > 0) {
            atomicAdd(&header->boulderPairs, (unsigned long long)warpBoulders);
        }
    }
}

// The compiled variants: (bin width, bin height, cells per thread).
constexpr BatchVariant kVariants[] = {
    {32, 32, 4}, {32, 32, 8}, {64, 32, 8}, {32, 16, 2}, {64, 64, 8},
};
constexpr int kVariantCount = int(sizeof(kVariants) / sizeof(kVariants[0]));

// The dynamic shared memory of a variant: per warp, 8 bytes per cell and its pair queue.
template <int kBinW, int kBinH, int kCells>
constexpr size_t dynamic_bytes() {
    constexpr size_t warps = size_t(kBinW) * kBinH / kCells / 32;
    return warps * 32 * kCells * sizeof(double) + warps * (31 + 32 * kCells) * sizeof(uint16_t);
}

// Lets the variant take its dynamic shared memory (set once, before any capture: occupancy()
// runs when a batch is planned).
template <int kBinW, int kBinH, int kCells, bool kFast>
cudaError_t allow_shared() {
    static const cudaError_t done = cudaFuncSetAttribute(
        batch_evaluate_kernel<kBinW, kBinH, kCells, kFast>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, int(dynamic_bytes<kBinW, kBinH, kCells>()));
    return done;
}

template <int kBinW, int kBinH, int kCells, bool kFast>
cudaError_t launch_variant(const CraterShapeKernel& k, const BatchNoise& noise,
                           const BatchView& v, uint32_t ctas, cudaStream_t stream) {
    if (cudaError_t err = allow_shared<kBinW, kBinH, kCells, kFast>()) {
        return err;
    }
    batch_evaluate_kernel<kBinW, kBinH, kCells, kFast>
        <<<ctas, kBinW * kBinH / kCells, dynamic_bytes<kBinW, kBinH, kCells>(), stream>>>(
            k, noise, v);
    return cudaGetLastError();
}

template <int kBinW, int kBinH, int kCells, bool kFast>
int occupancy() {
    int blocks = 0;
    if (allow_shared<kBinW, kBinH, kCells, kFast>() != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &blocks, batch_evaluate_kernel<kBinW, kBinH, kCells, kFast>, kBinW * kBinH / kCells,
            dynamic_bytes<kBinW, kBinH, kCells>()) != cudaSuccess) {
        return 1;
    }
    return blocks > 0 ? blocks : 1;
}

uint32_t grid_for(uint32_t items, uint32_t perBlock) {
    const uint64_t blocks = (uint64_t(items) + perBlock - 1) / perBlock;
    return uint32_t(blocks < 1 ? 1 : (blocks > 148u * 32u ? 148u * 32u : blocks));
}

}  // namespace

int batch_variant_count() {
    return kVariantCount;
}

BatchVariant batch_variant(int index) {
    return kVariants[index < 0 || index >= kVariantCount ? 0 : index];
}

int batch_blocks_per_sm(int index, bool fast) {
    if (!fast) {
        return occupancy<32, 32, 4, false>();
    }
    switch (index) {
        case 1: return occupancy<32, 32, 8, true>();
        case 2: return occupancy<64, 32, 8, true>();
        case 3: return occupancy<32, 16, 2, true>();
        case 4: return occupancy<64, 64, 8, true>();
        default: return occupancy<32, 32, 4, true>();
    }
}

cudaError_t launch_batch_bin(const CraterShapeKernel& k, const BatchView& v,
                             const BatchVariant& variant, uint32_t maxRecords,
                             uint32_t maxBoulders, uint32_t* scanScratch, cudaStream_t stream) {
    // maxRecords / maxBoulders: the (ref, record) and (ref, boulder) pairs the plan holds.
    const size_t words = size_t(v.capacityBins) + 1;
    cudaError_t err = cudaMemsetAsync(v.craterCounts, 0, words * sizeof(uint32_t), stream);
    if (err == cudaSuccess) {
        err = cudaMemsetAsync(v.craterCursor, 0, size_t(v.capacityBins) * sizeof(uint32_t), stream);
    }
    if (err == cudaSuccess) {
        err = cudaMemsetAsync(v.boulderCounts, 0, words * sizeof(uint32_t), stream);
    }
    if (err == cudaSuccess) {
        err = cudaMemsetAsync(v.boulderCursor, 0, size_t(v.capacityBins) * sizeof(uint32_t),
                              stream);
    }
    if (err != cudaSuccess) {
        return err;
    }
    const uint32_t tpbX = variant.binW / kRefTileCells, tpbY = variant.binH / kRefTileCells;
    if (maxRecords > 0) {
        batch_crater_count_kernel<<<grid_for(maxRecords, 256), 256, 0, stream>>>(k, v, tpbX,
                                                                                   tpbY);
        if ((err = cudaGetLastError()) != cudaSuccess) {
            return err;
        }
    }
    if (maxBoulders > 0) {
        batch_boulder_count_kernel<<<grid_for(maxBoulders, 256), 256, 0, stream>>>(
            v, variant.binW, variant.binH);
        if ((err = cudaGetLastError()) != cudaSuccess) {
            return err;
        }
    }
    if ((err = launch_exclusive_scan(v.craterCounts, v.capacityBins, scanScratch, stream)) !=
        cudaSuccess) {
        return err;
    }
    if ((err = launch_exclusive_scan(v.boulderCounts, v.capacityBins, scanScratch, stream)) !=
        cudaSuccess) {
        return err;
    }
    if (maxRecords > 0) {
        batch_crater_scatter_kernel<<<grid_for(maxRecords, 256), 256, 0, stream>>>(k, v, tpbX,
                                                                                     tpbY);
        if ((err = cudaGetLastError()) != cudaSuccess) {
            return err;
        }
        if (!v.harmonicsReady) {
            batch_harmonics_kernel<<<grid_for(maxRecords, 256), 256, 0, stream>>>(v);
            if ((err = cudaGetLastError()) != cudaSuccess) {
                return err;
            }
        }
    }
    if (maxBoulders > 0) {
        batch_boulder_scatter_kernel<<<grid_for(maxBoulders, 256), 256, 0, stream>>>(
            v, variant.binW, variant.binH);
        if ((err = cudaGetLastError()) != cudaSuccess) {
            return err;
        }
    }
    batch_totals_kernel<<<1, 1, 0, stream>>>(v);
    return cudaGetLastError();
}

cudaError_t batch_ds_setup(uint32_t& ctas) {
    static const cudaError_t allowed = [] {
        const int points = int(8 * kDsPointPool * sizeof(double));
        for (const auto& [kernel, bytes] :
             {std::make_pair(reinterpret_cast<const void*>(batch_ds_kernel<true>),
                             int(kDsSharedBudget)),
              std::make_pair(reinterpret_cast<const void*>(batch_ds_kernel<false>),
                             int(kDsSharedBudget)),
              std::make_pair(reinterpret_cast<const void*>(batch_ds_points_kernel<true>), points),
              std::make_pair(reinterpret_cast<const void*>(batch_ds_points_kernel<false>),
                             points)}) {
            const cudaError_t e =
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (e != cudaSuccess) {
                return e;
            }
        }
        return cudaSuccess;
    }();
    if (allowed != cudaSuccess) {
        return allowed;
    }
    int device = 0, sms = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err == cudaSuccess) {
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    }
    ctas = uint32_t(sms) * 3u;  // three CTAs of kDsSharedBudget node buffers share an SM
    return err;
}

cudaError_t launch_batch_ds(const BatchNoise& noise, const BatchView& v, bool spline,
                            uint32_t ctas, cudaStream_t stream) {
    const size_t bytes = kDsSharedBudget, points = 8 * kDsPointPool * sizeof(double);
    if (spline) {
        batch_ds_kernel<true><<<ctas, kDsTileThreads, bytes, stream>>>(noise, v);
        batch_ds_points_kernel<true><<<ctas, 256, points, stream>>>(noise, v);
    } else {
        batch_ds_kernel<false><<<ctas, kDsTileThreads, bytes, stream>>>(noise, v);
        batch_ds_points_kernel<false><<<ctas, 256, points, stream>>>(noise, v);
    }
    return cudaGetLastError();
}

cudaError_t launch_batch_evaluate(const CraterShapeKernel& k, const BatchNoise& noise,
                                  const BatchView& v, int variant, bool fast, uint32_t ctas,
                                  cudaStream_t stream) {
    if (!fast) {
        return launch_variant<32, 32, 4, false>(k, noise, v, ctas, stream);
    }
    switch (variant) {
        case 1: return launch_variant<32, 32, 8, true>(k, noise, v, ctas, stream);
        case 2: return launch_variant<64, 32, 8, true>(k, noise, v, ctas, stream);
        case 3: return launch_variant<32, 16, 2, true>(k, noise, v, ctas, stream);
        case 4: return launch_variant<64, 64, 8, true>(k, noise, v, ctas, stream);
        default: return launch_variant<32, 32, 4, true>(k, noise, v, ctas, stream);
    }
}

}  // namespace tgb
