// Boulder relief baking (BoulderLayer::ApplySamples with dome relief,
// src/layers/boulders/boulder_relief.cpp:426-439): each cell of each boulder's box gets
// max(height, base + weight * dome), base being the cell's height before the layer
// (DrawFeatures, include/terraingen/sources/sample_block.h:107-116) and the dome averaged over a
// sample width (DomeHeight, boulder_relief.cpp:44-57), in double as the reference computes it.
//
// Max-compositing is order-free: rounding to float is monotonic, so the result is
// float(max(height, max over boulders of base + weight * dome)) whatever order boulders come in,
// which lets them be binned by atomics. Launch structure as crater shaping (craters.cu): count,
// scan, scatter into kBinCells-square bins, then one CTA per bin stages its entries in shared
// memory by TMA bulk copies and each thread bakes 4 cells. A boulder touches the cells of its
// box's pixel window (ForEachFeatureCell, include/terraingen/raster/cell_loops.h:129-152).
#include "binning.cuh"
#include "kernels.h"

namespace tgb {
namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 4;
constexpr uint32_t kChunk = 96;  // 64-byte entries per staged chunk (6 KB)

using namespace binning;

__global__ void boulder_count_kernel(const BoulderRecord* __restrict__ boulders, uint32_t n,
                                     const Grid grid, double width, BoulderBins bins) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const BoulderRecord b = boulders[i];
    // ReliefBox on a plane (boulder_relief.cpp:24): reach 0.5 (diameter + width).
    const double reach = 0.5 * (b.diameter + width);
    int c0, c1, r0, r1;
    window_of(grid, b.x - reach, b.y - reach, b.x + reach, b.y + reach, c0, c1, r0, r1);
    const bool drawn = c0 < c1 && r0 < r1 && b.weight > 0.0;
    bins.windows[i] = drawn ? make_int4(c0, c1, r0, r1) : make_int4(1, 0, 1, 0);
    if (!drawn) {
        return;
    }
    const uint32_t bx0 = uint32_t(c0) / kBinCells, bx1 = uint32_t(c1 - 1) / kBinCells;
    const uint32_t by0 = uint32_t(r0) / kBinCells, by1 = uint32_t(r1 - 1) / kBinCells;
    for (uint32_t by = by0; by <= by1; ++by) {
        for (uint32_t bx = bx0; bx <= bx1; ++bx) {
            atomicAdd(bins.counts + by * bins.binsX + bx, 1u);
        }
    }
}

__global__ void boulder_scatter_kernel(const BoulderRecord* __restrict__ boulders, uint32_t n,
                                       BoulderBins bins) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !boulder_bins_usable(bins)) {
        return;
    }
    const int4 w = bins.windows[i];
    if (w.x >= w.y) {
        return;
    }
    const BoulderRecord b = boulders[i];
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
    const uint32_t bx0 = uint32_t(w.x) / kBinCells, bx1 = uint32_t(w.y - 1) / kBinCells;
    const uint32_t by0 = uint32_t(w.z) / kBinCells, by1 = uint32_t(w.w - 1) / kBinCells;
    for (uint32_t by = by0; by <= by1; ++by) {
        for (uint32_t bx = bx0; bx <= bx1; ++bx) {
            const uint32_t bin = by * bins.binsX + bx;
            const uint32_t slot = bins.counts[bin] + atomicAdd(bins.cursor + bin, 1u);
            if (slot < bins.capacity) {
                bins.entries[slot] = e;
            }
        }
    }
}

// Four CTAs per SM (64 registers a thread) to hide the bake's memory latencies.
__global__ void __launch_bounds__(kThreads, 4)
    boulder_bake_kernel(const Grid grid, const double width, const NoData nodata,
                        const BoulderBins bins, float* __restrict__ heights,
                        uint32_t* __restrict__ flags, const uint32_t polls) {
    __shared__ __align__(128) BoulderEntry stage[2][kChunk];
    __shared__ __align__(8) uint64_t bars[2];
    const uint32_t bin = bins.firstBin + blockIdx.x;
    if (!boulder_bins_usable(bins)) {
        // The entries were not scattered: nothing is baked, the host grows them and runs again.
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            atomicOr(flags, 4u);
        }
        return;
    }
    const uint32_t first = bins.counts[bin];
    const uint32_t count = bins.counts[bin + 1] - first;
    if (count == 0u) {
        return;
    }
    const uint32_t binX = bin % bins.binsX, binY = bin / bins.binsX;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const int row = int(binY * kBinCells + warp * 4u + lane / 8u);
    const int col0 = int(binX * kBinCells + (lane % 8u) * kCellsPerThread);
    const bool rowIn = row < int(grid.height);
    // Thread 0 starts the entry fetch before the cells' base heights are loaded, so the two
    // memory latencies overlap; the barrier after the loads publishes the mbarrier init.
    const uint32_t chunks = (count + kChunk - 1) / kChunk;
    auto issue = [&](uint32_t c) {
        const uint32_t s = c & 1u;
        const uint32_t bytes = min(kChunk, count - c * kChunk) * uint32_t(sizeof(BoulderEntry));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         smem_addr(&bars[s])),
                     "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(smem_addr(&stage[s][0])),
            "l"(bins.entries + first + c * kChunk), "r"(bytes), "r"(smem_addr(&bars[s]))
            : "memory");
    };
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        issue(0);
        if (chunks > 1) {
            issue(1);
        }
    }
    // Cell centers in double (Raster::CellCenter), the base heights and the running maxima.
    const double cy = grid.originY + (double(col0) + 0.5) * grid.colRotation +
                      (double(row) + 0.5) * grid.pixelHeight;
    double cx[kCellsPerThread], best[kCellsPerThread];
    float base[kCellsPerThread];
    bool live[kCellsPerThread];
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        const int col = col0 + j;
        cx[j] = grid.originX + (double(col) + 0.5) * grid.pixelWidth +
                (double(row) + 0.5) * grid.rowRotation;
        live[j] = rowIn && col < int(grid.width);
        base[j] = 0.0f;
        if (live[j]) {
            base[j] = heights[size_t(row) * grid.width + col];
            live[j] = !is_nodata(nodata, base[j]);
        }
        best[j] = double(base[j]);
    }
    __syncthreads();
    uint32_t phase[2] = {0u, 0u};
    uint32_t evaluated = 0;
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t s = c & 1u;
        const bool arrived = mbar_wait(&bars[s], phase[s], polls);
        if (__syncthreads_or(!arrived)) {
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
        for (uint32_t e = 0; e < n; ++e) {
            const BoulderEntry& b = stage[s][e];
            const bool inRows = row >= b.r0 && row < b.r1;
            bool any = false;
#pragma unroll
            for (int j = 0; j < kCellsPerThread; ++j) {
                any |= live[j] && inRows && col0 + j >= b.c0 && col0 + j < b.c1;
            }
            if (!__any_sync(0xffffffffu, any)) {
                continue;
            }
            const double dy = cy - b.y;
#pragma unroll
            for (int j = 0; j < kCellsPerThread; ++j) {
                if (live[j] && inRows && col0 + j >= b.c0 && col0 + j < b.c1) {
                    ++evaluated;
                    const double dx = cx[j] - b.x;
                    // RockRelief without facets: the dome, not below 0 (boulder.h:90-95).
                    const double relief = fmax(dome(b, hypot(dx, dy), width), 0.0);
                    if (relief > 0.0) {
                        best[j] = fmax(best[j], double(base[j]) + b.weight * relief);
                    }
                }
            }
        }
        __syncthreads();
        if (tid == 0 && c + 2 < chunks) {
            issue(c + 2);
        }
    }
    const uint32_t warpPairs = __reduce_add_sync(0xffffffffu, evaluated);
    if (lane == 0 && warpPairs > 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(flags + 2), (unsigned long long)warpPairs);
    }
    if (!rowIn) {
        return;
    }
    float* dst = heights + size_t(row) * grid.width + col0;
#pragma unroll
    for (int j = 0; j < kCellsPerThread; ++j) {
        if (live[j]) {
            dst[j] = float(best[j]);
        }
    }
}

}  // namespace

cudaError_t launch_boulder_count(const BoulderRecord* boulders, uint32_t n, const Grid& grid,
                                 double width, const BoulderBins& bins, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    boulder_count_kernel<<<(n + 255) / 256, 256, 0, stream>>>(boulders, n, grid, width, bins);
    return cudaGetLastError();
}

cudaError_t launch_boulder_scatter(const BoulderRecord* boulders, uint32_t n,
                                   const BoulderBins& bins, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    boulder_scatter_kernel<<<(n + 255) / 256, 256, 0, stream>>>(boulders, n, bins);
    return cudaGetLastError();
}

cudaError_t launch_boulder_bake(const Grid& grid, double width, NoData nodata,
                                const BoulderBins& bins, float* heights, uint32_t* flags,
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
    BoulderBins strip = bins;
    strip.firstBin = firstBinRow * bins.binsX;
    boulder_bake_kernel<<<nbins, kThreads, 0, stream>>>(grid, width, nodata, strip, heights,
                                                        flags, polls);
    return cudaGetLastError();
}

}  // namespace tgb
