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

// Each warp takes 32 craters: every lane finds its crater's footprint (its 16-cell tile window
// and cull radius, as CraterReach and TileLists give it), then the warp counts the bins of each
// crater in turn, its lanes spread over the crater's bins.
__global__ void crater_count_kernel(const CraterShapeKernel k, const CraterRecord* __restrict__ records,
                                    uint32_t n, const float* __restrict__ data,
                                    const double* __restrict__ footprints, const Grid grid,
                                    CraterBins bins, uint32_t* __restrict__ flags) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u;
    if (base >= n) {
        return;
    }
    const uint32_t mine = base + lane;
    int4 tiles = make_int4(1, 0, 1, 0);
    if (mine < n) {
        const CraterRecord r = records[mine];
        const Footprint f = crater_footprint(k, r, data, footprints, mine, grid);
        tiles = f.tiles;
        bins.boxes[mine] = tiles;
        bins.culls[mine] = f.cull;
        if (tiles.x <= tiles.y) {
            if (r.hasDatum == 1u) {
                atomicOr(flags, 1u);
            }
            // Anything beyond an ellipse and power-law harmonics, or a complex crater, needs
            // the general path.
            if (crater_entry_heavy(k, r)) {
                atomicOr(flags, 4u);
            }
        }
    }
    constexpr uint32_t kTilesPerBin = kBinCells / kRefTileCells;
    const uint32_t count = min(32u, n - base);
    for (uint32_t j = 0; j < count; ++j) {
        const int4 t = make_int4(__shfl_sync(0xffffffffu, tiles.x, int(j)),
                                 __shfl_sync(0xffffffffu, tiles.y, int(j)),
                                 __shfl_sync(0xffffffffu, tiles.z, int(j)),
                                 __shfl_sync(0xffffffffu, tiles.w, int(j)));
        if (t.x > t.y) {
            continue;
        }
        const uint32_t bx0 = uint32_t(t.x) / kTilesPerBin, bx1 = uint32_t(t.y) / kTilesPerBin;
        const uint32_t by0 = uint32_t(t.z) / kTilesPerBin, by1 = uint32_t(t.w) / kTilesPerBin;
        const uint32_t wide = bx1 - bx0 + 1u;
        const uint32_t total = wide * (by1 - by0 + 1u);
        for (uint32_t q = lane; q < total; q += 32u) {
            const uint32_t b = (by0 + q / wide) * bins.binsX + bx0 + q % wide;
            atomicAdd(bins.counts + b, 1u);
        }
    }
}

// Each warp takes 32 craters and spreads all of their (crater, bin) pairs over its lanes: a
// lane finds its pair's crater by a search of the warp's running bin counts, then copies the
// crater's record and tail into its bin's next slot.
__global__ void crater_scatter_kernel(const CraterShapeKernel k,
                                      const CraterRecord* __restrict__ records, uint32_t n,
                                      CraterBins bins) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u;
    if (base >= n) {
        return;
    }
    constexpr uint32_t kTilesPerBin = kBinCells / kRefTileCells;
    const uint32_t mine = base + lane;
    int4 tiles = make_int4(1, 0, 1, 0);
    float cull = 0.0f;
    uint32_t count = 0;
    if (mine < n) {
        tiles = bins.boxes[mine];
        cull = bins.culls[mine];
        if (tiles.x <= tiles.y) {
            count = (uint32_t(tiles.y) / kTilesPerBin - uint32_t(tiles.x) / kTilesPerBin + 1u) *
                    (uint32_t(tiles.w) / kTilesPerBin - uint32_t(tiles.z) / kTilesPerBin + 1u);
        }
    }
    // Inclusive running count of the warp's pairs.
    uint32_t upto = count;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, upto, d);
        if (lane >= uint32_t(d)) {
            upto += v;
        }
    }
    const uint32_t pairs = __shfl_sync(0xffffffffu, upto, 31);
    for (uint32_t q0 = 0; q0 < pairs; q0 += 32u) {
        const uint32_t q = q0 + lane;
        // The crater of pair q: the first lane whose running count exceeds q.
        uint32_t owner = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint32_t probe = owner + step - 1u;
            const uint32_t at = __shfl_sync(0xffffffffu, upto, int(probe));
            if (at <= q) {
                owner += step;
            }
        }
        const int4 t = make_int4(__shfl_sync(0xffffffffu, tiles.x, int(owner)),
                                 __shfl_sync(0xffffffffu, tiles.y, int(owner)),
                                 __shfl_sync(0xffffffffu, tiles.z, int(owner)),
                                 __shfl_sync(0xffffffffu, tiles.w, int(owner)));
        const float c = __shfl_sync(0xffffffffu, cull, int(owner));
        const uint32_t before = __shfl_sync(0xffffffffu, upto - count, int(owner));
        if (q >= pairs) {
            continue;
        }
        const uint32_t local = q - before;
        const uint32_t bx0 = uint32_t(t.x) / kTilesPerBin, bx1 = uint32_t(t.y) / kTilesPerBin;
        const uint32_t by0 = uint32_t(t.z) / kTilesPerBin;
        const uint32_t wide = bx1 - bx0 + 1u;
        const uint32_t b = (by0 + local / wide) * bins.binsX + bx0 + local % wide;
        const uint32_t slot = bins.counts[b] + atomicAdd(bins.cursor + b, 1u);
        if (slot >= bins.capacity) {
            continue;  // the host sized the entries from the counts; never taken
        }
        const uint32_t crater = base + owner;
        const int4* src = reinterpret_cast<const int4*>(records + crater);
        int4* dst = reinterpret_cast<int4*>(bins.entries + slot);
#pragma unroll
        for (int w = 0; w < 9; ++w) {
            dst[w] = __ldg(src + w);
        }
        const uint32_t heavy = crater_entry_heavy(k, records[crater]) ? kHeavyEntry : 0u;
        dst[9] = make_int4(int(uint32_t(t.x) | (uint32_t(t.y) << 16)),
                           int(uint32_t(t.z) | (uint32_t(t.w) << 16)), __float_as_int(c),
                           int(crater | heavy));
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
// one row). For every staged crater the warp first finds which of its 128 cells need it (inside
// a reference tile the crater's window touches, and within its cull radius), then queues those
// (crater, cell) pairs in shared memory and evaluates them 32 at a time, one pair per lane, so a
// small crater that needs a handful of cells no longer leaves most lanes of the warp idle. The
// contributions are FP32 values added into FP64 accumulators in shared memory: that sum is exact
// for these magnitudes, so the atomic adds give the same bits in any order.
//
// With kFast, entries marked kHeavyEntry (complex craters, peaks, terraces, tables) queue apart
// and are drained through the general contribution, so a batch with a few such craters keeps the
// lean path for all the others.
constexpr int kQueue = 160;  // 31 pairs left over plus one crater's 128

template <bool kFast>
__global__ void __launch_bounds__(kShapeThreads, kFast ? 2 : 1)
    crater_shape_kernel(const CraterShapeKernel k, const float* __restrict__ data,
                        const float* __restrict__ harmonics, const Grid grid, const NoData nodata,
                        const CraterBins bins, float* __restrict__ heights,
                        uint32_t* __restrict__ flags, const uint32_t polls) {
    __shared__ __align__(128) BinEntry stage[2][kChunk];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ double accs[kShapeThreads / 32][128];
    __shared__ uint16_t queues[kShapeThreads / 32][kQueue];
    __shared__ uint16_t heavyQueues[kShapeThreads / 32][kFast ? kQueue : 1];
    __shared__ float2 columns[kShapeThreads / 32][32];  // split x of the warp's 32 columns
    __shared__ float2 rows[kShapeThreads / 32][4];      // split y of its 4 rows

    const uint32_t bin = bins.firstBin + blockIdx.x;
    const uint32_t binX = bin % bins.binsX, binY = bin / bins.binsX;
    const uint32_t first = bins.counts[bin];
    const uint32_t count = bins.counts[bin + 1] - first;
    if (count == 0u) {
        return;
    }
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t row = binY * kBinCells + warp * 4u + lane / 8u;
    const uint32_t col0 = binX * kBinCells + (lane % 8u) * kCellsPerThread;
    double* acc = accs[warp];
    uint16_t* queue = queues[warp];
    uint16_t* heavyQueue = heavyQueues[warp];
    const uint32_t cell0 = (lane / 8u) * 32u + (lane % 8u) * kCellsPerThread;

    // This thread's cells: split positions (MakeSplitPoint, crater_kernel.cpp:303) of the
    // column centers at row 0 and the row center at column 0, as the reference's strips carry.
    float pxh[kCellsPerThread], pxl[kCellsPerThread];
    bool live[kCellsPerThread];
    const double yd = grid.originY + 0.5 * grid.colRotation + (double(row) + 0.5) * grid.pixelHeight;
    const float pyh = float(yd);
    const float pyl = float(yd - double(pyh));
    const bool rowIn = row < grid.height;
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        const uint32_t col = col0 + j;
        const double xd =
            grid.originX + (double(col) + 0.5) * grid.pixelWidth + 0.5 * grid.rowRotation;
        pxh[j] = float(xd);
        pxl[j] = float(xd - double(pxh[j]));
        live[j] = rowIn && col < grid.width;
        double h = 0.0;
        if (live[j]) {
            const float v = heights[size_t(row) * grid.width + col];
            live[j] = !is_nodata(nodata, v);
            h = double(v);
        }
        acc[cell0 + j] = h;
        if (lane < 8u) {
            columns[warp][(lane % 8u) * kCellsPerThread + j] = make_float2(pxh[j], pxl[j]);
        }
    }
    if (lane % 8u == 0u) {
        rows[warp][lane / 8u] = make_float2(pyh, pyl);
    }
    const int tileX = int(col0 / kRefTileCells), tileY = int(row / kRefTileCells);
    const bool anyLive = live[0] || live[1] || live[2] || live[3];
    // The warp's 4 x 32 cell centers as a box (axis-aligned grids): a crater whose cull circle
    // misses it, with a quarter cell to spare for rounding, needs none of the warp's cells, and
    // the warp passes it over at once (the same decision in every lane).
    const bool boxTest = grid.rowRotation == 0.0 && grid.colRotation == 0.0;
    const double boxX = grid.originX + (double(binX * kBinCells) + 16.0) * grid.pixelWidth;
    const double boxY = grid.originY + (double(binY * kBinCells + warp * 4u) + 2.0) * grid.pixelHeight;
    const float boxXh = float(boxX), boxXl = float(boxX - double(boxXh));
    const float boxYh = float(boxY), boxYl = float(boxY - double(boxYh));
    const float halfW = 15.75f * float(fabs(grid.pixelWidth));
    const float halfH = 1.75f * float(fabs(grid.pixelHeight));

    // Evaluates the 32 (or, at a flush, `n`) pairs queued in `q` from `from`, one per lane; the
    // general contribution when `general` (always without kFast).
    auto drain = [&](const BinEntry* chunk, const uint16_t* q, uint32_t from, uint32_t n,
                     bool general) {
        if (lane < n) {
            const uint32_t code = q[from + lane];
            const BinEntry& entry = chunk[code >> 7];
            const CraterRecord& r = entry.record;
            const uint32_t cell = code & 127u;
            const float2 cx = columns[warp][cell & 31u];
            const float2 cy = rows[warp][cell >> 5];
            const float dy = crater::split_difference(cy.x, cy.y, r.y, r.yLow);
            const float dx = crater::split_difference(cx.x, cx.y, r.x, r.xLow);
            if (kFast && !general) {
                bool reached;
                const float shaped =
                    crater::lean_contribution(k, harmonics, data, r, dx, dy, reached);
                if (reached) {
                    atomicAdd(acc + cell, double(shaped));
                }
            } else if (kFast) {
                const crater::Contribution q = crater::general_contribution(k, data, r, dx, dy);
                if (q.reached) {
                    atomicAdd(acc + cell, double(q.shaped));
                }
            } else {
                const crater::Contribution q = crater::crater_contribution(k, data, r, dx, dy);
                if (q.reached) {
                    atomicAdd(acc + cell, double(q.shaped));
                }
            }
        }
    };

    const uint32_t chunks = (count + kChunk - 1) / kChunk;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](uint32_t c) {
        const uint32_t s = c & 1u;
        const uint32_t n = min(kChunk, count - c * kChunk);
        const uint32_t bytes = n * uint32_t(sizeof(BinEntry));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bars[s], bytes);
        bulk_copy_g2s(&stage[s][0], bins.entries + first + c * kChunk, bytes, &bars[s]);
    };
    if (tid == 0) {
        issue(0);
        if (chunks > 1) {
            issue(1);
        }
    }
    uint32_t phase[2] = {0u, 0u};
    bool failed = false;
    uint32_t evaluated = 0;  // (cell, crater) pairs this warp queued, for the pair counter
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t s = c & 1u;
        if (!mbar_wait(&bars[s], phase[s], polls)) {
            failed = true;
        }
        if (__syncthreads_or(failed)) {
            // A copy did not land within `polls`: record it, then wait (bounded by the default
            // limit) for the copies still in flight into this buffer and the other one (chunk
            // c + 1 is issued by now), so no bulk copy is left writing into a finished CTA.
            if (tid == 0) {
                atomicOr(flags, 2u);
                mbar_wait(&bars[s], phase[s]);
                if (c + 1 < chunks) {
                    mbar_wait(&bars[s ^ 1u], phase[s ^ 1u]);
                }
            }
            return;
        }
        phase[s] ^= 1u;
        const uint32_t n = min(kChunk, count - c * kChunk);
        uint32_t queued = 0;       // warp-uniform
        uint32_t heavyQueued = 0;  // warp-uniform
        for (uint32_t e = 0; e < n; ++e) {
            const BinEntry& entry = stage[s][e];
            const CraterRecord& r = entry.record;
            if (boxTest) {
                const float gx = fmaxf(
                    fabsf(crater::split_difference(boxXh, boxXl, r.x, r.xLow)) - halfW, 0.0f);
                const float gy = fmaxf(
                    fabsf(crater::split_difference(boxYh, boxYl, r.y, r.yLow)) - halfH, 0.0f);
                if (gx * gx + gy * gy >= entry.cull * entry.cull) {
                    continue;  // warp-uniform
                }
            }
            const bool inTile = anyLive && tileX >= int(entry.tileX0) &&
                                tileX <= int(entry.tileX1) && tileY >= int(entry.tileY0) &&
                                tileY <= int(entry.tileY1);
            if (!__any_sync(0xffffffffu, inTile)) {
                continue;  // none of the warp's reference tiles is in the crater's window
            }
            const float dy = crater::split_difference(pyh, pyl, r.y, r.yLow);
            const float cull2 = entry.cull * entry.cull;
            uint32_t need = 0;
#pragma unroll
            for (int j = 0; j < kCellsPerThread; ++j) {
                const float dx = crater::split_difference(pxh[j], pxl[j], r.x, r.xLow);
                if (inTile && live[j] && dx * dx + dy * dy < cull2) {
                    need |= 1u << j;
                }
            }
            if (!__any_sync(0xffffffffu, need != 0u)) {
                continue;
            }
            const uint32_t mine = __popc(need);
            // Exclusive prefix of the lanes' counts.
            uint32_t before = mine;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, before, d);
                if (lane >= uint32_t(d)) {
                    before += v;
                }
            }
            const uint32_t total = __shfl_sync(0xffffffffu, before, 31);
            if (total == 0u) {
                continue;
            }
            before -= mine;
            const bool heavy = kFast && (entry.index & kHeavyEntry) != 0u;  // warp-uniform
            uint16_t* q = heavy ? heavyQueue : queue;
            uint32_t& length = heavy ? heavyQueued : queued;
            uint32_t slot = length + before;
            for (int j = 0; j < kCellsPerThread; ++j) {
                if (need & (1u << j)) {
                    q[slot++] = uint16_t((e << 7) | (cell0 + j));
                }
            }
            evaluated += mine;
            length += total;
            __syncwarp();
            while (length >= 32u) {
                length -= 32u;
                drain(stage[s], q, length, 32u, heavy);
                __syncwarp();
            }
        }
        if (queued > 0u) {
            drain(stage[s], queue, 0u, queued, false);
            __syncwarp();
        }
        if (kFast && heavyQueued > 0u) {
            drain(stage[s], heavyQueue, 0u, heavyQueued, true);
            __syncwarp();
        }
        if (c + 2 < chunks) {
            // The buffer is read by every warp before it is refilled.
            __syncthreads();
            if (tid == 0) {
                issue(c + 2);
            }
        }
    }
    // One atomic per warp: the pairs this CTA evaluated, into the 64-bit counter after the flags.
    const uint32_t warpPairs = __reduce_add_sync(0xffffffffu, evaluated);
    if (lane == 0 && warpPairs > 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(flags + 1), (unsigned long long)warpPairs);
    }
    __syncwarp();
    if (!rowIn) {
        return;
    }
    float out[kCellsPerThread];
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        out[j] = float(acc[cell0 + j]);
    }
    float* dst = heights + size_t(row) * grid.width + col0;
    const bool vec = (grid.width % 4u == 0u) && col0 + 3 < grid.width &&
                     ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0u) && live[0] && live[1] &&
                     live[2] && live[3];
    if (vec) {
        *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
        for (int j = 0; j < kCellsPerThread; ++j) {
            if (live[j]) {
                dst[j] = out[j];
            }
        }
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

cudaError_t launch_crater_count(const CraterShapeKernel& k, const CraterRecord* records,
                                uint32_t n, const float* data, const double* footprints,
                                const Grid& grid, const CraterBins& bins, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    const uint32_t threads = 256;  // 8 warps of 32 craters
    const uint32_t blocks = uint32_t((uint64_t(n) + threads - 1) / threads);
    crater_count_kernel<<<blocks, threads, 0, stream>>>(k, records, n, data, footprints, grid,
                                                        bins, bins.total + 1);
    return cudaGetLastError();
}

cudaError_t launch_crater_scatter(const CraterShapeKernel& k, const CraterRecord* records,
                                  uint32_t n, const Grid& grid, const CraterBins& bins,
                                  cudaStream_t stream) {
    (void)grid;
    if (n == 0) {
        return cudaSuccess;
    }
    const uint32_t threads = 256;  // 8 warps of 32 craters
    const uint32_t blocks = uint32_t((uint64_t(n) + threads - 1) / threads);
    crater_scatter_kernel<<<blocks, threads, 0, stream>>>(k, records, n, bins);
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

cudaError_t launch_crater_shape(const CraterShapeKernel& k, const float* data,
                                const float* harmonics, bool fast, const Grid& grid,
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
    if (fast) {
        crater_shape_kernel<true><<<nbins, kShapeThreads, 0, stream>>>(
            k, data, harmonics, grid, nodata, strip, heights, bins.total + 1, polls);
    } else {
        crater_shape_kernel<false><<<nbins, kShapeThreads, 0, stream>>>(
            k, data, harmonics, grid, nodata, strip, heights, bins.total + 1, polls);
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
