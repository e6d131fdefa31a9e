// Crater shaping over a grid (ApplyCraters, src/layers/craters/shaping/apply.cpp:339-376).
//
// Plain path, in four stream-ordered launches:
//   1. count   - one warp per crater: its footprint window on the grid, exactly as
//                CratersOnRaster / PixelWindowIn compute it (apply.cpp:225-237,
//                src/raster/cell_loops.cpp:21-28), turned into the range of the reference's
//                16-cell tiles it touches, and one count per kBinCells-square bin it covers;
//   2. scan    - exclusive prefix sum of the bin counts;
//   3. scatter - one warp per crater: a 160-byte BinEntry (record + tile range) into each bin;
//   4. shape   - one CTA per bin: the bin's entries are staged in shared memory by TMA bulk
//                copies (cp.async.bulk + mbarrier, double-buffered), each warp ballots whether
//                any of its cells needs a crater, and each thread adds the crater to its 4 cells
//                (one 16-byte store per thread at the end).
//
// Coverage matches the reference's: a crater is evaluated at every cell of each 16x16 tile its
// window touches (apply.cpp:119-143, 199-222), whatever the bin size here.
//
// Accumulation: without a datum a crater adds resolution * shaped relief independently of the
// height beneath it (apply_test.cpp:276-286), so the contributions are summed in an FP64
// accumulator. Each contribution is an FP32 value and the sum stays far inside 53 bits, so the
// accumulation is error-free: the result is the FP32 rounding of the exact sum, independent of
// the order atomics put the entries in, so every run gives the same bits.
#include "binning.cuh"
#include "crater_math.cuh"
#include "kernels.h"

namespace tgb {
namespace {

constexpr int kShapeThreads = 256;     // 8 warps; warp w covers rows 4w..4w+3 of a 32x32 bin
constexpr int kCellsPerThread = 4;     // 4 adjacent columns, one row
constexpr uint32_t kChunk = 96;        // entries per staged chunk (15 KB)

using namespace binning;

// Binning runs over (crater, bin) pairs, so a crater covering thousands of bins costs no more
// than as many small ones: the footprint pass finds each crater's tile box, cull radius and bin
// count; an exclusive scan of those counts numbers the pairs; the count and scatter passes take
// one pair per thread (grid-stride), each finding its crater by binary search in the scan.

// Per crater: its footprint (the 16-cell tile window and cull radius, as CraterReach and
// TileLists give it) and how many bins it covers, into pairStart[i] (scanned afterwards).
__global__ void crater_footprint_kernel(const CraterShapeKernel k,
                                        const CraterRecord* __restrict__ records, uint32_t n,
                                        const float* __restrict__ data,
                                        const double* __restrict__ footprints, const Grid grid,
                                        CraterBins bins, uint32_t* __restrict__ flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    constexpr uint32_t kTilesPerBin = kBinCells / kRefTileCells;
    const CraterRecord& r = records[i];
    const Footprint f = crater_footprint(k, r, data, footprints, i, grid);
    bins.boxes[i] = f.tiles;
    bins.culls[i] = f.cull;
    uint32_t pairs = 0;
    if (f.tiles.x <= f.tiles.y) {
        pairs = (uint32_t(f.tiles.y) / kTilesPerBin - uint32_t(f.tiles.x) / kTilesPerBin + 1u) *
                (uint32_t(f.tiles.w) / kTilesPerBin - uint32_t(f.tiles.z) / kTilesPerBin + 1u);
        if (r.hasDatum == 1u) {
            atomicOr(flags, 1u);
        }
        // Work for the extras pass after the lean kernel (heavy records, massif peaks).
        if (crater_needs_extras(k, r) || (crater_is_complex(k, r) && r.peakCount > 0u)) {
            atomicOr(flags, 4u);
        }
    }
    bins.pairStart[i] = pairs;
}

// The crater of pair p: the last crater whose first pair is at most p (pairStart scanned, with
// pairStart[n] the number of pairs).
__device__ __forceinline__ uint32_t pair_crater(const uint32_t* __restrict__ start, uint32_t n,
                                                uint32_t p) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= p) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Pair p's crater and bin.
__device__ __forceinline__ void pair_bin(const CraterBins& bins, uint32_t n, uint32_t p,
                                         uint32_t& crater, int4& tiles, uint32_t& bx,
                                         uint32_t& by) {
    constexpr uint32_t kTilesPerBin = kBinCells / kRefTileCells;
    crater = pair_crater(bins.pairStart, n, p);
    tiles = bins.boxes[crater];
    const uint32_t local = p - __ldg(bins.pairStart + crater);
    const uint32_t bx0 = uint32_t(tiles.x) / kTilesPerBin;
    const uint32_t wide = uint32_t(tiles.y) / kTilesPerBin - bx0 + 1u;
    bx = bx0 + local % wide;
    by = uint32_t(tiles.z) / kTilesPerBin + local / wide;
}

__global__ void crater_bin_count_kernel(uint32_t n, CraterBins bins) {
    const uint32_t pairs = bins.pairStart[n];
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pairs;
         p += gridDim.x * blockDim.x) {
        uint32_t crater, bx, by;
        int4 tiles;
        pair_bin(bins, n, p, crater, tiles, bx, by);
        atomicAdd(bins.counts + by * bins.binsX + bx, 1u);
    }
}

// Whether a massif peak of `radius` m around (x, y) can reach a cell center of bin (bx, by): the
// columns and rows of cell centers within the radius (a box, with a little slack) meet the bin's
// (rotated grids: always).
__device__ inline bool peak_meets_bin(const Grid& g, double x, double y, double radius,
                                      uint32_t bx, uint32_t by) {
    if (g.rowRotation != 0.0 || g.colRotation != 0.0) {
        return true;
    }
    const double px = (x - g.originX) / g.pixelWidth - 0.5;  // cell column whose center is at x
    const double py = (y - g.originY) / g.pixelHeight - 0.5;
    const double rx = radius / fabs(g.pixelWidth) * (1.0 + 1e-6) + 1e-6;
    const double ry = radius / fabs(g.pixelHeight) * (1.0 + 1e-6) + 1e-6;
    const double c0 = fmax(ceil(px - rx), double(bx * kBinCells));
    const double c1 = fmin(floor(px + rx), double(bx * kBinCells + kBinCells - 1u));
    const double r0 = fmax(ceil(py - ry), double(by * kBinCells));
    const double r1 = fmin(floor(py + ry), double(by * kBinCells + kBinCells - 1u));
    return c0 <= c1 && r0 <= r1;
}

// Each pair's entry in its bin's next slot. With `leans` the entries are crater indices, with
// kHeavyEntry where the extras pass has work (a heavy crater in all its bins, a massif peak in the
// bins its reach meets), and each such bin is listed once in bins.extrasList; otherwise they are
// BinEntry copies (the record and the tail).
__global__ void crater_bin_scatter_kernel(const CraterShapeKernel k,
                                          const CraterRecord* __restrict__ records, uint32_t n,
                                          const crater::LeanCrater* __restrict__ leans,
                                          const Grid grid, CraterBins bins) {
    if (!crater_bins_usable(bins)) {
        return;
    }
    const uint32_t pairs = bins.pairStart[n];
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pairs;
         p += gridDim.x * blockDim.x) {
        uint32_t crater, bx, by;
        int4 t;
        pair_bin(bins, n, p, crater, t, bx, by);
        const uint32_t b = by * bins.binsX + bx;
        const uint32_t slot = bins.counts[b] + atomicAdd(bins.cursor + b, 1u);
        if (slot >= bins.capacity) {
            continue;  // the total fits the capacity (checked above); never taken
        }
        const CraterRecord& r = records[crater];
        if (leans != nullptr) {
            bool extras = crater_needs_extras(k, r);
            if (!extras && crater_is_complex(k, r) && r.peakCount > 0u) {
                extras = peak_meets_bin(grid, double(r.x) + double(r.xLow),
                                        double(r.y) + double(r.yLow),
                                        sqrt(double(__ldg(&leans[crater].peakReach2))), bx, by);
            }
            reinterpret_cast<uint32_t*>(bins.entries)[slot] = crater | (extras ? kHeavyEntry : 0u);
            if (extras && atomicOr(bins.extrasMark + b, 1u) == 0u) {
                bins.extrasList[1u + atomicAdd(bins.extrasList, 1u)] = b;
            }
            continue;
        }
        const int4* src = reinterpret_cast<const int4*>(records + crater);
        int4* dst = reinterpret_cast<int4*>(bins.entries + slot);
#pragma unroll
        for (int w = 0; w < 9; ++w) {
            dst[w] = __ldg(src + w);
        }
        dst[9] = make_int4(int(uint32_t(t.x) | (uint32_t(t.y) << 16)),
                           int(uint32_t(t.z) | (uint32_t(t.w) << 16)),
                           __float_as_int(bins.culls[crater]), int(crater));
    }
}

// (amplitude, phase) of each record's outline harmonics as (amplitude cos phase,
// amplitude sin phase), at the same offsets, for the lean path (crater_math.cuh).
__global__ void crater_harmonics_kernel(const CraterRecord* __restrict__ records, uint32_t n,
                                        const float* __restrict__ data, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint32_t offset = records[i].harmonicOffset;
    const uint32_t count = records[i].harmonicCount;
    for (uint32_t h = 0; h < count; ++h) {
        const float amplitude = __ldg(data + offset + 2u * h);
        const float phase = __ldg(data + offset + 2u * h + 1u);
        float s, c;
        sincosf(phase, &s, &c);
        out[offset + 2u * h] = amplitude * c;
        out[offset + 2u * h + 1u] = amplitude * s;
    }
}

// Shaping a bin. Each warp owns 4 rows x 32 columns of the bin (each thread 4 adjacent cells of
// one row). For every staged crater the warp first finds which of its 128 cells need it (within
// its cull radius, and for stretched craters inside a reference tile its window touches), then
// queues those (crater, cell) pairs in shared memory and evaluates them 32 at a time, one pair
// per lane, so a small crater that needs a handful of cells does not leave most lanes of the
// warp idle.
//
// Accumulation is in 64-bit fixed point (2^-32 m): each contribution is rounded once to a
// multiple of 2^-32 m and the integers are summed, which is exact and associative, so the bins'
// atomically scattered entry order cannot change a bit; the cell's height is the float of its
// height before the layer plus that sum. The warp owns its 128 accumulators, so lanes of one
// drain that land on different cells never collide; lanes on the same cell add atomically.
constexpr int kQueue = 160;  // 31 pairs left over plus one crater's 128
constexpr float kFixedScale = 4294967296.0f;  // 2^32 per meter
constexpr double kFixedUnit = 1.0 / 4294967296.0;

__device__ __forceinline__ long long to_fixed(float v) {
    return __float2ll_rn(v * kFixedScale);
}

__device__ __forceinline__ void add_fixed(long long* acc, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(acc), static_cast<unsigned long long>(v));
}

// The cells a warp owns and their split positions (MakeSplitPoint, crater_kernel.cpp:303: the
// column centers at row 0 and the row center at column 0, as the reference's strips carry them).
struct WarpCells {
    uint32_t row, col0, cell0;
    bool rowIn;
    bool live[kCellsPerThread];
    float base[kCellsPerThread];
    float pxh[kCellsPerThread], pxl[kCellsPerThread];
    float pyh, pyl;
    int tileX, tileY;
    bool anyLive;
};

__device__ __forceinline__ WarpCells warp_cells(const Grid& grid, const NoData& nodata,
                                                const float* __restrict__ heights, uint32_t binX,
                                                uint32_t binY, uint32_t warp, uint32_t lane) {
    WarpCells w;
    w.row = binY * kBinCells + warp * 4u + lane / 8u;
    w.col0 = binX * kBinCells + (lane % 8u) * kCellsPerThread;
    w.cell0 = (lane / 8u) * 32u + (lane % 8u) * kCellsPerThread;
    const double yd =
        grid.originY + 0.5 * grid.colRotation + (double(w.row) + 0.5) * grid.pixelHeight;
    w.pyh = float(yd);
    w.pyl = float(yd - double(w.pyh));
    w.rowIn = w.row < grid.height;
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        const uint32_t col = w.col0 + j;
        const double xd =
            grid.originX + (double(col) + 0.5) * grid.pixelWidth + 0.5 * grid.rowRotation;
        w.pxh[j] = float(xd);
        w.pxl[j] = float(xd - double(w.pxh[j]));
        w.live[j] = w.rowIn && col < grid.width;
        w.base[j] = 0.0f;
        if (w.live[j]) {
            w.base[j] = heights[size_t(w.row) * grid.width + col];
            w.live[j] = !is_nodata(nodata, w.base[j]);
        }
    }
    w.tileX = int(w.col0 / kRefTileCells);
    w.tileY = int(w.row / kRefTileCells);
    w.anyLive = w.live[0] || w.live[1] || w.live[2] || w.live[3];
    return w;
}

// The cell-center box of a warp's 4 x 32 cells on an axis-aligned grid, with a quarter cell to
// spare for rounding: a crater whose cull circle misses it needs none of the warp's cells.
struct WarpBox {
    float xh, xl, yh, yl, halfW, halfH;
    bool on;
};

__device__ __forceinline__ WarpBox warp_box(const Grid& grid, uint32_t binX, uint32_t binY,
                                            uint32_t warp) {
    WarpBox b;
    b.on = grid.rowRotation == 0.0 && grid.colRotation == 0.0;
    const double x = grid.originX + (double(binX * kBinCells) + 16.0) * grid.pixelWidth;
    const double y = grid.originY + (double(binY * kBinCells + warp * 4u) + 2.0) * grid.pixelHeight;
    b.xh = float(x);
    b.xl = float(x - double(b.xh));
    b.yh = float(y);
    b.yl = float(y - double(b.yh));
    b.halfW = 15.75f * float(fabs(grid.pixelWidth));
    b.halfH = 1.75f * float(fabs(grid.pixelHeight));
    return b;
}

__device__ __forceinline__ bool box_misses(const WarpBox& b, float x, float xLow, float y,
                                           float yLow, float cull) {
    if (!b.on) {
        return false;
    }
    const float gx = fmaxf(fabsf(crater::split_difference(b.xh, b.xl, x, xLow)) - b.halfW, 0.0f);
    const float gy = fmaxf(fabsf(crater::split_difference(b.yh, b.yl, y, yLow)) - b.halfH, 0.0f);
    return gx * gx + gy * gy >= cull * cull;
}

// The lane's cells that need a crater at (x, y) within `cull`, as bits.
__device__ __forceinline__ uint32_t need_mask(const WarpCells& w, bool inTile, float x,
                                              float xLow, float y, float yLow, float cull) {
    const float dy = crater::split_difference(w.pyh, w.pyl, y, yLow);
    const float cull2 = cull * cull;
    uint32_t need = 0;
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        const float dx = crater::split_difference(w.pxh[j], w.pxl[j], x, xLow);
        if (inTile && w.live[j] && dx * dx + dy * dy < cull2) {
            need |= 1u << j;
        }
    }
    return need;
}

// Appends the lanes' needed pairs (entry e, cell) to the warp's queue; returns how many.
__device__ __forceinline__ uint32_t enqueue(uint16_t* queue, uint32_t length, uint32_t need,
                                            uint32_t e, uint32_t cell0, uint32_t lane) {
    const uint32_t mine = __popc(need);
    uint32_t before = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, before, d);
        if (lane >= uint32_t(d)) {
            before += v;
        }
    }
    const uint32_t total = __shfl_sync(0xffffffffu, before, 31);
    uint32_t slot = length + before - mine;
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        if (need & (1u << j)) {
            queue[slot++] = uint16_t((e << 7) | (cell0 + j));
        }
    }
    return total;
}

// Writes a thread's cells: base height plus the fixed-point sum, one 16-byte store when it can.
__device__ __forceinline__ void write_cells(const Grid& grid, const WarpCells& w,
                                            const long long* acc, float* __restrict__ heights) {
    if (!w.rowIn) {
        return;
    }
    float out[kCellsPerThread];
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        out[j] = float(double(w.base[j]) + double(acc[w.cell0 + j]) * kFixedUnit);
    }
    float* dst = heights + size_t(w.row) * grid.width + w.col0;
    const bool vec = (grid.width % 4u == 0u) && w.col0 + 3 < grid.width &&
                     ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0u) && w.live[0] &&
                     w.live[1] && w.live[2] && w.live[3];
    if (vec) {
        *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
        for (int j = 0; j < kCellsPerThread; ++j) {
            if (w.live[j]) {
                dst[j] = out[j];
            }
        }
    }
}

// The staged-copy pipeline of a bin's entries: two shared buffers, each filled by one TMA bulk
// copy completing on its mbarrier. On a wait that gives up (`polls`) it records flag 2 and waits,
// bounded by the default limit, for the copies still in flight, so none lands in a finished CTA.
template <typename Entry, uint32_t kStage>
struct Stager {
    Entry (*stage)[kStage];
    uint64_t* bars;
    const Entry* src;
    uint32_t count, chunks, phase[2];

    __device__ void issue(uint32_t c) {
        const uint32_t s = c & 1u;
        const uint32_t n = min(kStage, count - c * kStage);
        const uint32_t bytes = n * uint32_t(sizeof(Entry));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bars[s], bytes);
        bulk_copy_g2s(&stage[s][0], src + c * kStage, bytes, &bars[s]);
    }

    // Thread 0 only: inits the barriers and starts the first two chunks.
    __device__ void start() {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issue(0);
        if (chunks > 1) {
            issue(1);
        }
    }

    // Every thread: waits for chunk c; false (after the drain) when it did not arrive.
    __device__ bool wait(uint32_t c, uint32_t polls, uint32_t* flags) {
        const uint32_t s = c & 1u;
        const bool failed = !mbar_wait(&bars[s], phase[s], polls);
        if (__syncthreads_or(failed)) {
            if (threadIdx.x == 0) {
                atomicOr(flags, 2u);
                mbar_wait(&bars[s], phase[s]);
                if (c + 1 < chunks) {
                    mbar_wait(&bars[s ^ 1u], phase[s ^ 1u]);
                }
            }
            return false;
        }
        phase[s] ^= 1u;
        return true;
    }

    // After every warp has read chunk c: its buffer takes chunk c + 2.
    __device__ void refill(uint32_t c) {
        if (c + 2 < chunks) {
            __syncthreads();
            if (threadIdx.x == 0) {
                issue(c + 2);
            }
        }
    }
};

// The general binned kernel: any kernel options and any record, from the 160-byte BinEntry.
__global__ void __launch_bounds__(kShapeThreads)
    crater_shape_kernel(const CraterShapeKernel k, const float* __restrict__ data,
                        const Grid grid, const NoData nodata, const CraterBins bins,
                        float* __restrict__ heights, uint32_t* __restrict__ flags,
                        const uint32_t polls) {
    __shared__ __align__(128) BinEntry stage[2][kChunk];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ long long accs[kShapeThreads / 32][128];
    __shared__ uint16_t queues[kShapeThreads / 32][kQueue];
    __shared__ float2 columns[kShapeThreads / 32][32];
    __shared__ float2 rows[kShapeThreads / 32][4];

    const uint32_t bin = bins.firstBin + blockIdx.x;
    const uint32_t binX = bin % bins.binsX, binY = bin / bins.binsX;
    const uint32_t first = bins.counts[bin];
    const uint32_t count = bins.counts[bin + 1] - first;
    if (count == 0u || !crater_bins_usable(bins)) {
        return;
    }
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    Stager<BinEntry, kChunk> st{stage, bars, bins.entries + first, count,
                                (count + kChunk - 1) / kChunk, {0u, 0u}};
    if (tid == 0) {
        st.start();
    }
    const WarpCells w = warp_cells(grid, nodata, heights, binX, binY, warp, lane);
    const WarpBox box = warp_box(grid, binX, binY, warp);
    long long* acc = accs[warp];
    uint16_t* queue = queues[warp];
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        acc[w.cell0 + j] = 0;
        if (lane < 8u) {
            columns[warp][(lane % 8u) * kCellsPerThread + j] = make_float2(w.pxh[j], w.pxl[j]);
        }
    }
    if (lane % 8u == 0u) {
        rows[warp][lane / 8u] = make_float2(w.pyh, w.pyl);
    }
    __syncthreads();

    auto drain = [&](const BinEntry* chunk, uint32_t from, uint32_t n) {
        if (lane < n) {
            const uint32_t code = queue[from + lane];
            const CraterRecord& r = chunk[code >> 7].record;
            const uint32_t cell = code & 127u;
            const float2 cx = columns[warp][cell & 31u];
            const float2 cy = rows[warp][cell >> 5];
            const float dy = crater::split_difference(cy.x, cy.y, r.y, r.yLow);
            const float dx = crater::split_difference(cx.x, cx.y, r.x, r.xLow);
            const crater::Contribution q = crater::crater_contribution(k, data, r, dx, dy);
            if (q.reached) {
                add_fixed(acc + cell, to_fixed(q.shaped));
            }
        }
    };

    uint32_t evaluated = 0;
    for (uint32_t c = 0; c < st.chunks; ++c) {
        if (!st.wait(c, polls, flags)) {
            return;
        }
        const uint32_t s = c & 1u;
        const uint32_t n = min(kChunk, count - c * kChunk);
        uint32_t queued = 0;  // warp-uniform
        for (uint32_t e = 0; e < n; ++e) {
            const BinEntry& entry = stage[s][e];
            const CraterRecord& r = entry.record;
            if (box_misses(box, r.x, r.xLow, r.y, r.yLow, entry.cull)) {
                continue;  // warp-uniform
            }
            const bool inTile = w.anyLive && w.tileX >= int(entry.tileX0) &&
                                w.tileX <= int(entry.tileX1) && w.tileY >= int(entry.tileY0) &&
                                w.tileY <= int(entry.tileY1);
            const uint32_t need = need_mask(w, inTile, r.x, r.xLow, r.y, r.yLow, entry.cull);
            if (!__any_sync(0xffffffffu, need != 0u)) {
                continue;
            }
            evaluated += __popc(need);
            queued += enqueue(queue, queued, need, e, w.cell0, lane);
            __syncwarp();
            while (queued >= 32u) {
                queued -= 32u;
                drain(stage[s], queued, 32u);
                __syncwarp();
            }
        }
        if (queued > 0u) {
            drain(stage[s], 0u, queued);
            __syncwarp();
        }
        st.refill(c);
    }
    const uint32_t warpPairs = __reduce_add_sync(0xffffffffu, evaluated);
    if (lane == 0 && warpPairs > 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(flags + 1), (unsigned long long)warpPairs);
    }
    __syncwarp();
    write_cells(grid, w, acc, heights);
}

// Each crater's LeanCrater (crater_math.cuh), made once after the count pass.
__global__ void crater_lean_kernel(const CraterShapeKernel k,
                                   const CraterRecord* __restrict__ records, uint32_t n,
                                   const float* __restrict__ data, const CraterBins bins,
                                   crater::LeanCrater* __restrict__ leans) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        leans[i] = crater::lean_crater(k, records[i], data, i, bins.boxes[i], bins.culls[i]);
    }
}

constexpr uint32_t kLeanChunk = 64;  // 13 KB a buffer

// The lean kernel's staging: a bin holds crater indices, and warp 0 gathers each chunk's
// LeanCraters into a shared buffer with one 208-byte TMA bulk copy per entry, all completing on
// the buffer's mbarrier (lane 0 arrives with the chunk's byte count before any copy is issued).
// Waits give up after `polls`, record flag 2 and drain the copies in flight, as Stager's do.
struct LeanStager {
    crater::LeanCrater (*stage)[kLeanChunk];
    uint64_t* bars;
    const uint32_t* indices;
    const crater::LeanCrater* leans;
    uint32_t count, chunks, phase[2];

    // Warp 0 only.
    __device__ void issue(uint32_t c, uint32_t lane) {
        const uint32_t s = c & 1u;
        const uint32_t n = min(kLeanChunk, count - c * kLeanChunk);
        if (lane == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bars[s], n * uint32_t(sizeof(crater::LeanCrater)));
        }
        __syncwarp();
        for (uint32_t e = lane; e < n; e += 32u) {
            const uint32_t index = __ldg(indices + c * kLeanChunk + e) & ~kHeavyEntry;
            bulk_copy_g2s(&stage[s][e], leans + index, uint32_t(sizeof(crater::LeanCrater)),
                          &bars[s]);
        }
    }

    // Warp 0 only: inits the barriers and starts the first two chunks.
    __device__ void start(uint32_t lane) {
        if (lane == 0) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
        issue(0, lane);
        if (chunks > 1) {
            issue(1, lane);
        }
    }

    __device__ bool wait(uint32_t c, uint32_t polls, uint32_t* flags) {
        const uint32_t s = c & 1u;
        const bool failed = !mbar_wait(&bars[s], phase[s], polls);
        if (__syncthreads_or(failed)) {
            if (threadIdx.x == 0) {
                atomicOr(flags, 2u);
                mbar_wait(&bars[s], phase[s]);
                if (c + 1 < chunks) {
                    mbar_wait(&bars[s ^ 1u], phase[s ^ 1u]);
                }
            }
            return false;
        }
        phase[s] ^= 1u;
        return true;
    }

    __device__ void refill(uint32_t c, uint32_t warp, uint32_t lane) {
        if (c + 2 < chunks) {
            __syncthreads();
            if (warp == 0) {
                issue(c + 2, lane);
            }
        }
    }
};

// The lean binned kernel (plain kernel options): each pair through `lean_contribution`; heavy
// craters and massif peaks are left to the extras pass. Four CTAs of 256 threads per SM (64
// registers, no spills; three CTAs at 71 registers were 7 % slower).
__global__ void __launch_bounds__(kShapeThreads, 4)
    crater_lean_shape_kernel(const CraterShapeKernel k, const CraterRecord* __restrict__ records,
                             const float* __restrict__ data,
                             const crater::LeanCrater* __restrict__ leans, const Grid grid,
                             const NoData nodata, const CraterBins bins,
                             float* __restrict__ heights, uint32_t* __restrict__ flags,
                             const uint32_t polls) {
    __shared__ __align__(128) crater::LeanCrater stage[2][kLeanChunk];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ long long accs[kShapeThreads / 32][128];
    __shared__ uint16_t queues[kShapeThreads / 32][kQueue];
    __shared__ float2 columns[kShapeThreads / 32][32];
    __shared__ float2 rows[kShapeThreads / 32][4];
    __shared__ WarpBox boxes[kShapeThreads / 32];
    __shared__ uint8_t warpMasks[2][kLeanChunk];  // per staged crater: the warps it can touch

    const uint32_t bin = bins.firstBin + blockIdx.x;
    const uint32_t binX = bin % bins.binsX, binY = bin / bins.binsX;
    const uint32_t first = bins.counts[bin];
    const uint32_t count = bins.counts[bin + 1] - first;
    if (count == 0u || !crater_bins_usable(bins)) {
        return;
    }
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    LeanStager st{stage, bars, reinterpret_cast<const uint32_t*>(bins.entries) + first, leans,
                  count, (count + kLeanChunk - 1) / kLeanChunk, {0u, 0u}};
    if (warp == 0) {
        st.start(lane);
    }
    const WarpCells w = warp_cells(grid, nodata, heights, binX, binY, warp, lane);
    long long* acc = accs[warp];
    uint16_t* queue = queues[warp];
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        acc[w.cell0 + j] = 0;
        if (lane < 8u) {
            columns[warp][(lane % 8u) * kCellsPerThread + j] = make_float2(w.pxh[j], w.pxl[j]);
        }
    }
    if (lane % 8u == 0u) {
        rows[warp][lane / 8u] = make_float2(w.pyh, w.pyl);
    }
    if (lane == 0) {
        boxes[warp] = warp_box(grid, binX, binY, warp);
    }
    const crater::LeanKernel lk = crater::lean_kernel(k);
    __syncthreads();

    auto drain = [&](const crater::LeanCrater* chunk, uint32_t from, uint32_t n) {
        if (lane < n) {
            const uint32_t code = queue[from + lane];
            const crater::LeanCrater& l = chunk[code >> 7];
            const uint32_t cell = code & 127u;
            const float2 cx = columns[warp][cell & 31u];
            const float2 cy = rows[warp][cell >> 5];
            const float4 center = *reinterpret_cast<const float4*>(&l.x);  // x, xLow, y, yLow
            const float dy = crater::split_difference(cy.x, cy.y, center.z, center.w);
            const float dx = crater::split_difference(cx.x, cx.y, center.x, center.y);
            bool reached;
            float shaped;
            const float v = crater::lean_contribution(k, lk, l, dx, dy, reached, shaped);
            if (reached) {
                add_fixed(acc + cell, to_fixed(v));
            }
        }
    };

    uint32_t evaluated = 0;
    for (uint32_t c = 0; c < st.chunks; ++c) {
        if (!st.wait(c, polls, flags)) {
            return;
        }
        const uint32_t s = c & 1u;
        const uint32_t n = min(kLeanChunk, count - c * kLeanChunk);
        // Which warps' cell boxes each staged crater's cull circle meets, one thread a crater
        // (heavy craters are the extras pass's: none). The masks are double-buffered like the
        // stage: the wait before chunk c + 2 is a block barrier, so chunk c's are read by then.
        if (tid < n) {
            const crater::LeanCrater& l = stage[s][tid];
            uint32_t mask = 0;
            if (!(l.flags & crater::kLeanHeavy)) {
#pragma unroll
                for (uint32_t v = 0; v < kShapeThreads / 32; ++v) {
                    if (!box_misses(boxes[v], l.x, l.xLow, l.y, l.yLow, l.cull)) {
                        mask |= 1u << v;
                    }
                }
            }
            warpMasks[s][tid] = uint8_t(mask);
        }
        __syncthreads();
        uint32_t queued = 0;  // warp-uniform
        for (uint32_t e = 0; e < n; ++e) {
            // A lean crater is never stretched, so every cell within its cull radius lies inside
            // its footprint window: no tile test.
            if (((warpMasks[s][e] >> warp) & 1u) == 0u) {
                continue;  // warp-uniform
            }
            const crater::LeanCrater& l = stage[s][e];
            const uint32_t need = need_mask(w, true, l.x, l.xLow, l.y, l.yLow, l.cull);
            if (!__any_sync(0xffffffffu, need != 0u)) {
                continue;
            }
            evaluated += __popc(need);
            queued += enqueue(queue, queued, need, e, w.cell0, lane);
            __syncwarp();
            while (queued >= 32u) {
                queued -= 32u;
                drain(stage[s], queued, 32u);
                __syncwarp();
            }
        }
        if (queued > 0u) {
            drain(stage[s], 0u, queued);
            __syncwarp();
        }
        st.refill(c, warp, lane);
    }
    const uint32_t warpPairs = __reduce_add_sync(0xffffffffu, evaluated);
    if (lane == 0 && warpPairs > 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(flags + 1), (unsigned long long)warpPairs);
    }
    __syncwarp();
    write_cells(grid, w, acc, heights);
}

// The extras pass after the lean kernel: heavy craters (tables, marks, terraces, shifts,
// upslopes, long outlines) through the general contribution, and the massif peaks' difference
// from the round dome the lean pass gave their craters, in the bins the scatter listed
// (bins.extrasList) and only those of this launch's strip of bin rows. Rare work: each CTA takes
// listed bins in turn, each thread evaluates its own 4 cells against each flagged entry of the
// bin, read from global memory, and adds the fixed-point sum to the heights the lean pass wrote.
__global__ void __launch_bounds__(kShapeThreads)
    crater_extras_kernel(const CraterShapeKernel k, const CraterRecord* __restrict__ records,
                         const float* __restrict__ data,
                         const crater::LeanCrater* __restrict__ leans, const Grid grid,
                         const NoData nodata, const CraterBins bins, uint32_t binsInStrip,
                         float* __restrict__ heights) {
    if ((bins.total[1] & 4u) == 0u || !crater_bins_usable(bins)) {
        return;  // no heavy record nor massif peak in the layer
    }
    const uint32_t listed = bins.extrasList[0];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t item = blockIdx.x; item < listed; item += gridDim.x) {
        const uint32_t bin = bins.extrasList[1u + item];
        if (bin < bins.firstBin || bin >= bins.firstBin + binsInStrip) {
            continue;  // block-uniform: another strip's bin
        }
        const uint32_t binX = bin % bins.binsX, binY = bin / bins.binsX;
        const uint32_t first = bins.counts[bin];
        const uint32_t count = bins.counts[bin + 1] - first;
        const uint32_t* indices = reinterpret_cast<const uint32_t*>(bins.entries) + first;
        const WarpCells w = warp_cells(grid, nodata, heights, binX, binY, warp, lane);
        long long sum[kCellsPerThread] = {0, 0, 0, 0};
        for (uint32_t e = 0; e < count; ++e) {
            const uint32_t index = __ldg(indices + e);
            if ((index & kHeavyEntry) == 0u) {
                continue;  // block-uniform
            }
            const uint32_t c = index & ~kHeavyEntry;
            const crater::LeanCrater& l = leans[c];
            const CraterRecord& r = records[c];
            const uint32_t lflags = __ldg(&l.flags);
            float cull = __ldg(&l.cull);
            bool inTile = true;
            if (lflags & crater::kLeanHeavy) {
                inTile = w.anyLive && w.tileX >= int(__ldg(&l.tileX0)) &&
                         w.tileX <= int(__ldg(&l.tileX1)) && w.tileY >= int(__ldg(&l.tileY0)) &&
                         w.tileY <= int(__ldg(&l.tileY1));
            } else {
                cull = sqrtf(__ldg(&l.peakReach2)) * (1.0f + 1e-5f) + 1e-6f;  // the massif peak's
            }
            const uint32_t need = need_mask(w, inTile, r.x, r.xLow, r.y, r.yLow, cull);
            if (need == 0u) {
                continue;
            }
            const float dy = crater::split_difference(w.pyh, w.pyl, r.y, r.yLow);
#pragma unroll
            for (int j = 0; j < kCellsPerThread; ++j) {
                if (need & (1u << j)) {
                    const float dx = crater::split_difference(w.pxh[j], w.pxl[j], r.x, r.xLow);
                    bool reached;
                    const float v =
                        crater::extra_contribution(k, data, r, lflags, dx, dy, reached);
                    if (reached) {
                        sum[j] += to_fixed(v);
                    }
                }
            }
        }
        if (w.rowIn) {
            float* dst = heights + size_t(w.row) * grid.width + w.col0;
#pragma unroll
            for (int j = 0; j < kCellsPerThread; ++j) {
                if (w.live[j] && sum[j] != 0) {
                    dst[j] = float(double(w.base[j]) + double(sum[j]) * kFixedUnit);
                }
            }
        }
        __syncthreads();  // the next bin's cells are read only after this one's are written
    }
}

// The drop-in form: cell by cell over its tile's ordered crater list, in float, as
// ShapeTilesOnCpu / craters.slang do (apply.cpp:199-222, src/layers/kernels/craters.slang).
__global__ void crater_shape_lists_kernel(const CraterShapeKernel k,
                                          const CraterRecord* __restrict__ records,
                                          const float* __restrict__ data,
                                          const uint32_t* __restrict__ heads,
                                          const uint32_t* __restrict__ entries, uint32_t width,
                                          uint32_t rows, uint32_t firstRow,
                                          const float* __restrict__ xs,
                                          const float* __restrict__ xLows,
                                          const float* __restrict__ ys,
                                          const float* __restrict__ yLows, const NoData nodata,
                                          float* __restrict__ heights) {
    const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= width || r >= rows) {
        return;
    }
    const size_t i = size_t(r) * width + col;
    float height = heights[i];
    if (is_nodata(nodata, height)) {
        return;
    }
    const uint32_t row = firstRow + r;
    const uint32_t side = heads[1];
    const uint32_t head = 3u + 2u * ((row / side) * heads[0] + col / side);
    const uint32_t first = heads[head], n = heads[head + 1];
    const float px = xs[col], pxl = xLows[col], py = ys[r], pyl = yLows[row];
    for (uint32_t e = first; e < first + n; ++e) {
        const CraterRecord& c = records[entries[e]];
        const float dx = crater::split_difference(px, pxl, c.x, c.xLow);
        const float dy = crater::split_difference(py, pyl, c.y, c.yLow);
        const crater::Contribution q = crater::crater_contribution(k, data, c, dx, dy);
        if (!q.reached) {
            continue;
        }
        height = c.hasDatum == 1u ? crater::apply_with_datum(c, q, height, dx, dy)
                                  : height + q.shaped;
    }
    heights[i] = height;
}

// The same on a body (ShapeCratersOnBody, craters.h:1360; craters.slang's body branch): each
// cell's position is a split point in 3D and each crater is read in its frame, the offset
// projected on the crater's tangent plane (azimuthal equidistant on a sphere, KernelFrameOffset).
__global__ void crater_shape_body_kernel(const CraterShapeKernel k,
                                         const CraterRecord* __restrict__ records,
                                         const CraterFrame* __restrict__ frames,
                                         const float* __restrict__ data,
                                         const uint32_t* __restrict__ heads,
                                         const uint32_t* __restrict__ entries, uint32_t width,
                                         uint32_t rows, uint32_t firstRow,
                                         const SplitPoint* __restrict__ points,
                                         const NoData nodata, float* __restrict__ heights) {
    const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= width || r >= rows) {
        return;
    }
    const size_t i = size_t(r) * width + col;
    float height = heights[i];
    if (is_nodata(nodata, height)) {
        return;
    }
    const uint32_t row = firstRow + r;
    const uint32_t side = heads[1];
    const uint32_t head = 3u + 2u * ((row / side) * heads[0] + col / side);
    const uint32_t first = heads[head], n = heads[head + 1];
    const SplitPoint p = points[i];
    for (uint32_t e = first; e < first + n; ++e) {
        const uint32_t m = entries[e];
        const CraterRecord& c = records[m];
        const CraterFrame& f = frames[m];
        const crater::Offset at =
            crater::frame_offset(f, crater::split_difference(p.x, p.xLow, f.x, f.xLow),
                                 crater::split_difference(p.y, p.yLow, f.y, f.yLow),
                                 crater::split_difference(p.z, p.zLow, f.z, f.zLow));
        const crater::Contribution q = crater::crater_contribution(k, data, c, at.dx, at.dy);
        if (!q.reached) {
            continue;
        }
        height = c.hasDatum == 1u ? crater::apply_with_datum(c, q, height, at.dx, at.dy)
                                  : height + q.shaped;
    }
    heights[i] = height;
}

// --- exclusive scan ------------------------------------------------------------------------

constexpr uint32_t kScanBlock = 1024;

__global__ void scan_block_kernel(uint32_t* data, uint32_t n, uint32_t* blockSums) {
    __shared__ uint32_t warpSums[32];
    const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    const uint32_t v = i < n ? data[i] : 0u;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) {
            x += y;
        }
    }
    if (lane == 31u) {
        warpSums[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warpSums[lane];
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) {
                w += y;
            }
        }
        warpSums[lane] = w;
    }
    __syncthreads();
    const uint32_t before = (warp > 0 ? warpSums[warp - 1] : 0u) + x - v;
    if (i < n) {
        data[i] = before;
    }
    if (threadIdx.x == kScanBlock - 1) {
        blockSums[blockIdx.x] = warpSums[31];
    }
}

__global__ void scan_add_kernel(uint32_t* data, uint32_t n, const uint32_t* blockOffsets) {
    const uint32_t i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) {
        data[i] += blockOffsets[blockIdx.x];
    }
}

}  // namespace

size_t scan_scratch_words(uint32_t n) {
    // Mirrors launch_exclusive_scan: n + 1 values in blocks of kScanBlock, one block sum each plus
    // the slot the next level's total lands in, recursively.
    const uint32_t blocks = (n + 1 + kScanBlock - 1) / kScanBlock;
    return size_t(blocks) + 1 + (blocks > 1 ? scan_scratch_words(blocks) : 0);
}

// In place over counts[0..n); counts[n] receives the total.
cudaError_t launch_exclusive_scan(uint32_t* counts, uint32_t n, uint32_t* scratch,
                                  cudaStream_t stream) {
    // Scanning n + 1 values leaves the total of the first n at index n.
    const uint32_t m = n + 1;
    const uint32_t blocks = (m + kScanBlock - 1) / kScanBlock;
    scan_block_kernel<<<blocks, kScanBlock, 0, stream>>>(counts, m, scratch);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess || blocks == 1) {
        return err;
    }
    // Block sums -> block offsets, recursively (blocks + 1 entries with the total last).
    err = cudaMemsetAsync(scratch + blocks, 0, sizeof(uint32_t), stream);
    if (err != cudaSuccess) {
        return err;
    }
    err = launch_exclusive_scan(scratch, blocks, scratch + blocks + 1, stream);
    if (err != cudaSuccess) {
        return err;
    }
    scan_add_kernel<<<blocks, kScanBlock, 0, stream>>>(counts, m, scratch);
    return cudaGetLastError();
}

// Grid of the pair-parallel passes (grid-stride over the pairs, whose number stays on the device).
constexpr uint32_t kPairBlocks = 148u * 8u;

cudaError_t launch_crater_count(const CraterShapeKernel& k, const CraterRecord* records,
                                uint32_t n, const float* data, const double* footprints,
                                const Grid& grid, const CraterBins& bins, uint32_t* scratch,
                                cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    crater_footprint_kernel<<<(n + 255) / 256, 256, 0, stream>>>(k, records, n, data, footprints,
                                                                 grid, bins, bins.total + 1);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        err = launch_exclusive_scan(bins.pairStart, n, scratch, stream);
    }
    if (err != cudaSuccess) {
        return err;
    }
    crater_bin_count_kernel<<<kPairBlocks, 256, 0, stream>>>(n, bins);
    return cudaGetLastError();
}

cudaError_t launch_crater_scatter(const CraterShapeKernel& k, const CraterRecord* records,
                                  uint32_t n, const Grid& grid, const CraterBins& bins,
                                  const void* leans, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    crater_bin_scatter_kernel<<<kPairBlocks, 256, 0, stream>>>(
        k, records, n, static_cast<const crater::LeanCrater*>(leans), grid, bins);
    return cudaGetLastError();
}

cudaError_t launch_crater_lean(const CraterShapeKernel& k, const CraterRecord* records, uint32_t n,
                               const float* data, const CraterBins& bins, void* leans,
                               cudaStream_t stream) {
    static_assert(sizeof(crater::LeanCrater) == kLeanCraterBytes, "lean crater size");
    if (n == 0) {
        return cudaSuccess;
    }
    crater_lean_kernel<<<(n + 127) / 128, 128, 0, stream>>>(
        k, records, n, data, bins, static_cast<crater::LeanCrater*>(leans));
    return cudaGetLastError();
}

cudaError_t launch_crater_harmonics(const CraterRecord* records, uint32_t n, const float* data,
                                    float* harmonics, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    crater_harmonics_kernel<<<(n + 255) / 256, 256, 0, stream>>>(records, n, data, harmonics);
    return cudaGetLastError();
}

bool crater_fast_path(const CraterShapeKernel& k, uint32_t batchFlags) {
    const CraterProfileKernel& p = k.profile;
    return (batchFlags & 4u) == 0u &&
           (p.simple == kProfileFassettThomson || p.simple == kProfileMartinParkesDunstan) &&
           p.complex == 0u && p.diffused == 0u && k.rimSigma == 0.0f &&
           k.noiseAmplitude == 0.0f && k.noiseRimAmplitude == 0.0f && k.wallStreaks == 0.0f &&
           k.ejecta == 0.0f;
}

bool crater_lean_entries(const CraterShapeKernel& k) {
    return crater_options_plain(k);
}

cudaError_t launch_crater_shape(const CraterShapeKernel& k, const CraterRecord* records,
                                const float* data, const void* leans, bool extras,
                                const Grid& grid,
                                NoData nodata, const CraterBins& bins, float* heights,
                                cudaStream_t stream, uint32_t firstBinRow, uint32_t binRows,
                                uint32_t polls) {
    if (firstBinRow >= bins.binsY) {
        return cudaSuccess;
    }
    const uint32_t rowsRun = std::min(binRows, bins.binsY - firstBinRow);
    const uint32_t nbins = bins.binsX * rowsRun;
    if (nbins == 0) {
        return cudaSuccess;
    }
    CraterBins strip = bins;
    strip.firstBin = firstBinRow * bins.binsX;
    if (leans != nullptr) {
        const auto* lean = static_cast<const crater::LeanCrater*>(leans);
        crater_lean_shape_kernel<<<nbins, kShapeThreads, 0, stream>>>(
            k, records, data, lean, grid, nodata, strip, heights, bins.total + 1, polls);
        if (extras) {
            const cudaError_t err = cudaGetLastError();
            if (err != cudaSuccess) {
                return err;
            }
            const uint32_t grid2 = std::min(nbins, 148u * 4u);
            crater_extras_kernel<<<grid2, kShapeThreads, 0, stream>>>(
                k, records, data, lean, grid, nodata, strip, nbins, heights);
        }
    } else {
        crater_shape_kernel<<<nbins, kShapeThreads, 0, stream>>>(k, data, grid, nodata, strip,
                                                                 heights, bins.total + 1, polls);
    }
    return cudaGetLastError();
}

cudaError_t launch_crater_shape_lists(const CraterShapeKernel& k, const CraterRecord* records,
                                      const float* data, const uint32_t* heads,
                                      const uint32_t* entries, uint32_t width, uint32_t rows,
                                      uint32_t firstRow, const float* xs, const float* xLows,
                                      const float* ys, const float* yLows, NoData nodata,
                                      float* heights, cudaStream_t stream) {
    if (width == 0 || rows == 0) {
        return cudaSuccess;
    }
    const dim3 block(16, 16);
    const dim3 blocks((width + 15) / 16, (rows + 15) / 16);
    crater_shape_lists_kernel<<<blocks, block, 0, stream>>>(k, records, data, heads, entries,
                                                            width, rows, firstRow, xs, xLows, ys,
                                                            yLows, nodata, heights);
    return cudaGetLastError();
}

cudaError_t launch_crater_shape_body(const CraterShapeKernel& k, const CraterRecord* records,
                                     const CraterFrame* frames, const float* data,
                                     const uint32_t* heads, const uint32_t* entries,
                                     uint32_t width, uint32_t rows, uint32_t firstRow,
                                     const SplitPoint* points, const NoData& nodata,
                                     float* heights, cudaStream_t stream) {
    const dim3 block(16, 16);
    const dim3 grid((width + 15) / 16, (rows + 15) / 16);
    crater_shape_body_kernel<<<grid, block, 0, stream>>>(k, records, frames, data, heads, entries,
                                                         width, rows, firstRow, points, nodata,
                                                         heights);
    return cudaGetLastError();
}

}  // namespace tgb
