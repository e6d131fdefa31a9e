// Diamond-square refinement of a DEM (DiamondSquareUpsampler::FillSamples,
// src/sources/diamond_square.cpp:426-516): posts refined `levels` times, each level halving the
// node spacing by a square step (odd/odd nodes: mean of the four parents plus a displacement) and
// a diamond step (mixed nodes: mean of the four neighbors plus a displacement), then read
// bilinearly at every output cell.
//
// Nodes are doubles, as in the reference. One CTA per output block builds the block's node
// pyramid in shared memory, every level over the box the next one reads (worked out top-down
// from the block's cells, as Refine's recursion does with its margins), and writes only the
// block's heights: no level touches HBM. Node values do not depend on the box they are computed
// in (displacements keyed by (seed, node, level) through Philox4x32-10, local means), so blocks
// agree on the nodes they share, and on the reference's.
//
// Compiled with -fmad=false, so the means and the read-out round as the reference's; the normal
// draws are float Box-Muller on exact double uniforms (node_normal).
#include <algorithm>
#include <cmath>

#include "ds_tile.cuh"

namespace tgb {
namespace {

template <bool kSpline>
__global__ void __launch_bounds__(kDsTileThreads) ds_tile_kernel(const DsTile t) {
    extern __shared__ double pool[];
    __shared__ DsShared sh;
    const PostsFromArray posts{t.posts, t.col0, t.row0, t.pw, t.ph};
    ds_block<kSpline>(t, blockIdx.x, posts, t.heights, pool, sh);
}

__global__ void philox_probe_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                    uint32_t* __restrict__ out, double* __restrict__ normals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint32_t* c = in + 6 * i;
    const Words w = philox(Words{c[0], c[1], c[2], c[3]}, c[4], c[5]);
    out[4 * i] = w.x;
    out[4 * i + 1] = w.y;
    out[4 * i + 2] = w.z;
    out[4 * i + 3] = w.w;
    // The displacement normal of node (c0, c1) at level c2 & 31 with seed c4, as signed 32-bit
    // node indices.
    normals[i] = node_normal(int64_t(int32_t(c[0])), int64_t(int32_t(c[1])), int(c[2] & 31u), c[4]);
}


// The output block of a diamond-square CTA and the shared buffers its node pyramid needs: the
// largest block (64 x 64, 64 x 32, 32 x 32, ... cells; one cell for a point) whose two buffers
// fit kDsSharedBudget bytes, so that three CTAs share an SM. A bigger block recomputes fewer nodes of its neighbours'
// (the margins the means need) per cell. Each level's box is bounded from the block's extent in
// finest nodes (what the device works out, plus two nodes for the rounding of either side's
// arithmetic), then level by level: the box the diamond step reads grows by the mean's reach, and
// its parents' box is half of it plus the square mean's margins.

bool ds_tile_shape(DsTile& t, bool spline, bool single) {
    const int64_t reach = spline ? 3 : 1, before = spline ? 1 : 0, after = spline ? 2 : 1;
    const Grid& g = t.grid;
    constexpr uint32_t kShapes[][2] = {{64, 64}, {64, 32}, {32, 32}, {32, 16}, {16, 16}, {16, 8},
                                       {8, 8},   {8, 4},   {4, 4},   {4, 2},   {2, 2},   {1, 1}};
    for (const auto& shape : kShapes) {
        const uint32_t bw = single ? 1u : shape[0], bh = single ? 1u : shape[1];
        const double spanX = (double(bw - 1) * std::fabs(g.pixelWidth) +
                              double(bh - 1) * std::fabs(g.rowRotation)) /
                             std::fabs(t.frame.stepX);
        const double spanY = (double(bw - 1) * std::fabs(g.colRotation) +
                              double(bh - 1) * std::fabs(g.pixelHeight)) /
                             std::fabs(t.frame.stepY);
        if (!(spanX < 4096.0 && spanY < 4096.0)) {
            continue;
        }
        int64_t w = int64_t(std::floor(spanX)) + 6 + after;
        int64_t h = int64_t(std::floor(spanY)) + 6 + after;
        uint64_t cap[2] = {0, 0};
        for (int l = t.levels; l >= 1; --l) {
            const int64_t ow = w + 2 * reach, oh = h + 2 * reach;
            cap[l & 1] = std::max<uint64_t>(cap[l & 1], uint64_t(ow * oh));
            w = ow / 2 + before + after + 1;
            h = oh / 2 + before + after + 1;
        }
        cap[0] = std::max<uint64_t>(cap[0], uint64_t(w * h));
        if ((cap[0] + cap[1]) * sizeof(double) <= kDsSharedBudget) {
            t.blockW = bw;
            t.blockH = bh;
            t.blocksX = (g.width + bw - 1) / bw;
            t.capEven = uint32_t(cap[0]);
            t.capOdd = uint32_t(cap[1]);
            return true;
        }
    }
    return false;
}


}  // namespace

bool ds_setup(DsTile& t, const Grid& pg, double fractalDimension, double scale, uint32_t seed,
              double minPixelSize, bool spline, const Grid& g, bool single) {
    // Levels(post spacing, spacing) (diamond_square.cpp:289-300).
    const double postSpacing = std::max(std::fabs(pg.pixelWidth), std::fabs(pg.pixelHeight));
    const double spacing = std::max(std::fabs(g.pixelWidth), std::fabs(g.pixelHeight));
    const double ratio = postSpacing / spacing;
    int levels = 0;
    if (ratio > 1.0) {
        double most = 30.0;
        if (minPixelSize > 0.0) {
            most = std::min(std::max(std::floor(std::log2(postSpacing / minPixelSize) + 1e-9), 0.0),
                            30.0);
        }
        levels = int(std::min(std::ceil(std::log2(ratio) - 1e-9), most));
    }
    // Frame (diamond_square.cpp:299-306): post (0, 0)'s center and the finest node steps.
    t.grid = g;
    t.frame.originX = pg.originX + 0.5 * pg.pixelWidth + 0.5 * pg.rowRotation;
    t.frame.originY = pg.originY + 0.5 * pg.colRotation + 0.5 * pg.pixelHeight;
    t.frame.stepX = std::ldexp(pg.pixelWidth, -levels);
    t.frame.stepY = std::ldexp(-pg.pixelHeight, -levels);
    t.levels = levels;
    t.seed = seed;
    // Displacement scales per level (Refinement::Displacement, diamond_square.cpp:382-389).
    const double stepFactor = std::pow(2.0, -(3.0 - fractalDimension) / 2.0);
    for (int l = 1; l <= levels; ++l) {
        t.squareStep[l] = scale * std::pow(stepFactor, 2 * l - 1);
        t.diamondStep[l] = scale * std::pow(stepFactor, 2 * l);
    }
    t.pitch = g.width;
    if (!ds_tile_shape(t, spline, single)) {
        return false;
    }
    t.blocks = t.blocksX * ((g.height + t.blockH - 1) / t.blockH);
    return true;
}

cudaError_t launch_ds_tiles(const DsTile& t, bool spline, cudaStream_t stream) {
    const uint32_t blocks = t.blocksX * ((t.grid.height + t.blockH - 1) / t.blockH);
    if (blocks == 0) {
        return cudaSuccess;
    }
    const size_t bytes = size_t(t.capEven + t.capOdd) * sizeof(double);
    cudaError_t err;
    if (spline) {
        err = cudaFuncSetAttribute(ds_tile_kernel<true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (err == cudaSuccess) {
            ds_tile_kernel<true><<<blocks, kDsTileThreads, bytes, stream>>>(t);
        }
    } else {
        err = cudaFuncSetAttribute(ds_tile_kernel<false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (err == cudaSuccess) {
            ds_tile_kernel<false><<<blocks, kDsTileThreads, bytes, stream>>>(t);
        }
    }
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_philox_probe(const uint32_t* in, uint32_t n, uint32_t* out, double* normals,
                                cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    philox_probe_kernel<<<(n + 127) / 128, 128, 0, stream>>>(in, n, out, normals);
    return cudaGetLastError();
}

}  // namespace tgb
