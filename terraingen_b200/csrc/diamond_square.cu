// Diamond-square refinement of a DEM (DiamondSquareUpsampler::FillSamples,
// src/sources/diamond_square.cpp:426-516): posts refined `levels` times, each level halving the
// node spacing by a square step (odd/odd nodes: mean of the four parents plus a displacement) and
// a diamond step (mixed nodes: mean of the four neighbors plus a displacement), then read
// bilinearly at every output cell.
//
// Nodes are doubles, as in the reference, materialised level by level in HBM over boxes that
// contain what the next level reads (worked out top-down from the output grid, as Refine's
// recursion does with its margins). Node values do not depend on the box they are computed in:
// displacements are keyed by (seed, node, level) through Philox4x32-10 and means are local, which
// is what lets the GPU compute every node once instead of recomputing parents per tile.
//
// Compiled with -fmad=false, so the means and the read-out round as the reference's; the normal
// draws are float Box-Muller on exact double uniforms (node_normal).
#include "kernels.h"

namespace tgb {
namespace {

constexpr uint32_t kMidpointDisplacementStream = 0x524D4450u;  // streams.h:73

struct Words {
    uint32_t x, y, z, w;
};

// Philox4x32-10 (include/terraingen/random/philox.h:43-91).
__device__ __forceinline__ Words philox(Words c, uint32_t k0, uint32_t k1) {
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

// The standard normal of node (col, row) of `level` (Refinement::Displacement,
// diamond_square.cpp:382-389): one Philox block is RandomStream's first two NextDouble draws
// (u1, u2, 53 bits each, exact), turned into a normal by Box-Muller (StandardNormal,
// src/random/samplers.cpp:65-69), sqrt(-2 log(1 - u1)) cos(2 pi u2). The reference evaluates it
// in double; here the logarithm, the square root and the cosine run in float on arguments formed
// exactly in double, within 2e-6 of the double normal (a few 1e-7 of the radius; under 1e-5 m in
// the refined heights) for a fraction of the instructions: the steps are bound by issuing them.
__device__ __forceinline__ double node_normal(int64_t col, int64_t row, int level,
                                              uint32_t seed) {
    const uint32_t high = uint32_t((col >> 32) ^ (row >> 32));
    const Words b = philox(Words{uint32_t(col), uint32_t(row), uint32_t(level) | (high << 5), 0u},
                           seed, kMidpointDisplacementStream);
    const double u1 =
        double((uint64_t(b.x >> 5u) << 26u) | uint64_t(b.y >> 6u)) * 0x1p-53;
    const double u2 =
        double((uint64_t(b.z >> 5u) << 26u) | uint64_t(b.w >> 6u)) * 0x1p-53;
    // log(1 - u1): log1p of the float u1 while it is small, else log of the float 1 - u1 (exact
    // in double), each a few 1e-8 relative.
    const float logRest = u1 < 0.5 ? log1pf(-float(u1)) : logf(float(1.0 - u1));
    const float radius = sqrtf(-2.0f * logRest);
    // cos(pi a) for a = 2 u2 split into float parts a = high + low: cos(pi high) - pi low
    // sin(pi high), so the float rounding of a costs no accuracy.
    const double a = 2.0 * u2;
    const float aHigh = float(a), aLow = float(a - double(aHigh));
    float sine, cosine;
    sincospif(aHigh, &sine, &cosine);
    const float c = fmaf(-3.14159265f * aLow, sine, cosine);
    return double(radius) * double(c);
}

__device__ __forceinline__ double at(const DsLevel& l, int64_t col, int64_t row) {
    return l.nodes[size_t(row - l.r0) * l.w + size_t(col - l.c0)];
}

// Catmull-Rom weights of four nodes around a midpoint (diamond_square.cpp:37).
__device__ __constant__ const double kMid[4] = {-1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0, -1.0 / 16.0};

// Level 0: node (col, row) is post (col, -row), reads past the held posts repeating their edge
// (BaseNodes, diamond_square.cpp:308; PostIndex, src/sources/lattice.h:99). The `pw` x `ph`
// posts held are those of columns [col0, col0 + pw) and rows [row0, row0 + ph) of the lattice.
__global__ void ds_base_kernel(const float* __restrict__ posts, int64_t col0, int64_t row0,
                               uint32_t pw, uint32_t ph, DsLevel out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= out.w || j >= out.h) {
        return;
    }
    const int64_t col = out.c0 + i - col0, row = -(out.r0 + j) - row0;
    const int64_t pc = col < 0 ? 0 : (col >= int64_t(pw) ? int64_t(pw) - 1 : col);
    const int64_t pr = row < 0 ? 0 : (row >= int64_t(ph) ? int64_t(ph) - 1 : row);
    out.nodes[size_t(j) * out.w + i] = double(posts[size_t(pr) * pw + size_t(pc)]);
}

// Nodes are handled in 2 x 2 blocks anchored at even (col, row): every thread of a step draws
// the same number of normals (one in the square step, two in the diamond step), so no lane of
// a warp idles while the others run Philox and Box-Muller.

// The square step of `level` over `out`'s box: kept parents (even/even) and displaced odd/odd
// nodes (SquareStep, diamond_square.cpp:392-407), block (bc0 + i, br0 + j) per thread. Mixed
// nodes are left for the diamond step.
template <bool kSpline>
__global__ void ds_square_kernel(const DsLevel parents, DsLevel out, int64_t bc0, int64_t br0,
                                 uint32_t bw, uint32_t bh, int level, double step,
                                 uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= bw || j >= bh) {
        return;
    }
    const int64_t bc = bc0 + i, br = br0 + j;
    const int64_t c1 = out.c0 + int64_t(out.w), r1 = out.r0 + int64_t(out.h);
    // The kept parent at (2 bc, 2 br).
    const int64_t ec = 2 * bc, er = 2 * br;
    if (ec >= out.c0 && ec < c1 && er >= out.r0 && er < r1) {
        out.nodes[size_t(er - out.r0) * out.w + size_t(ec - out.c0)] = at(parents, bc, br);
    }
    // The displaced node at (2 bc + 1, 2 br + 1): the mean of the four parents around it.
    const int64_t col = ec + 1, row = er + 1;
    if (col < out.c0 || col >= c1 || row < out.r0 || row >= r1) {
        return;
    }
    const int64_t left = bc, bottom = br;
    double mean;
    if (!kSpline) {
        mean = 0.25 * (at(parents, left, bottom) + at(parents, left + 1, bottom) +
                       at(parents, left, bottom + 1) + at(parents, left + 1, bottom + 1));
    } else {
        mean = 0.0;
        for (int64_t b = 0; b < 4; ++b) {
            double line = 0.0;
            for (int64_t a = 0; a < 4; ++a) {
                line += kMid[a] * at(parents, left - 1 + a, bottom - 1 + b);
            }
            mean += kMid[b] * line;
        }
    }
    out.nodes[size_t(row - out.r0) * out.w + size_t(col - out.c0)] =
        mean + step * node_normal(col, row, level, seed);
}

// A mixed node (col, row) of the diamond step: the mean of the four square-step nodes around it
// plus its displacement.
template <bool kSpline>
__device__ __forceinline__ void diamond_node(DsLevel& nodes, int64_t col, int64_t row, int level,
                                             double step, uint32_t seed) {
    double mean;
    if (!kSpline) {
        mean = 0.25 * (at(nodes, col - 1, row) + at(nodes, col + 1, row) + at(nodes, col, row - 1) +
                       at(nodes, col, row + 1));
    } else {
        double alongX = 0.0, alongY = 0.0;
        for (int64_t k = 0; k < 4; ++k) {
            alongX += kMid[k] * at(nodes, col - 3 + 2 * k, row);
            alongY += kMid[k] * at(nodes, col, row - 3 + 2 * k);
        }
        mean = 0.5 * (alongX + alongY);
    }
    nodes.nodes[size_t(row - nodes.r0) * nodes.w + size_t(col - nodes.c0)] =
        mean + step * node_normal(col, row, level, seed);
}

// The diamond step of `level`: the mixed nodes (2 bc + 1, 2 br) and (2 bc, 2 br + 1) of block
// (bc0 + i, br0 + j) that lie in `box` (inner box of `nodes`), from the square step's nodes
// around them (DiamondStep, diamond_square.cpp:410-424).
template <bool kSpline>
__global__ void ds_diamond_kernel(DsLevel nodes, int64_t c0, int64_t r0, uint32_t w, uint32_t h,
                                  int64_t bc0, int64_t br0, uint32_t bw, uint32_t bh, int level,
                                  double step, uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= bw || j >= bh) {
        return;
    }
    const int64_t bc = bc0 + i, br = br0 + j;
    const int64_t c1 = c0 + int64_t(w), r1 = r0 + int64_t(h);
    const int64_t cols[2] = {2 * bc + 1, 2 * bc}, rows[2] = {2 * br, 2 * br + 1};
    for (int n = 0; n < 2; ++n) {
        if (cols[n] >= c0 && cols[n] < c1 && rows[n] >= r0 && rows[n] < r1) {
            diamond_node<kSpline>(nodes, cols[n], rows[n], level, step, seed);
        }
    }
}

// `value` as an integer when within 1e-6 of one (NearestWhole, src/sources/lattice.h:33), else
// the node below and the share of the way to the next (NodeAndShare, diamond_square.cpp:53).
__device__ __forceinline__ void node_and_share(double u, int64_t& node, double& share) {
    const double rounded = round(u);
    if (fabs(u - rounded) <= 1e-6) {
        node = int64_t(rounded);
        share = 0.0;
        return;
    }
    const double below = floor(u);
    node = int64_t(below);
    share = u - below;
}

// Bilinear read of the finest nodes at every cell of the output grid (Interpolate,
// diamond_square.cpp:461-485).
__global__ void ds_read_kernel(const DsLevel nodes, DsFrame frame, const Grid grid,
                               float* __restrict__ heights) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= grid.width || r >= grid.height) {
        return;
    }
    const double x = grid.originX + (double(c) + 0.5) * grid.pixelWidth +
                     (double(r) + 0.5) * grid.rowRotation;
    const double y = grid.originY + (double(c) + 0.5) * grid.colRotation +
                     (double(r) + 0.5) * grid.pixelHeight;
    int64_t col, row;
    double u, v;
    node_and_share((x - frame.originX) / frame.stepX, col, u);
    node_and_share((y - frame.originY) / frame.stepY, row, v);
    double value = at(nodes, col, row);
    if (u > 0.0) {
        value = value * (1.0 - u) + at(nodes, col + 1, row) * u;
    }
    if (v > 0.0) {
        double above = at(nodes, col, row + 1);
        if (u > 0.0) {
            above = above * (1.0 - u) + at(nodes, col + 1, row + 1) * u;
        }
        value = value * (1.0 - v) + above * v;
    }
    heights[size_t(r) * grid.width + c] = float(value);
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

dim3 blocks_for(uint32_t w, uint32_t h, dim3 block) {
    return dim3((w + block.x - 1) / block.x, (h + block.y - 1) / block.y);
}

}  // namespace

cudaError_t launch_ds_base(const float* posts, int64_t col0, int64_t row0, uint32_t pw,
                           uint32_t ph, const DsLevel& out, cudaStream_t stream) {
    const dim3 block(32, 8);
    ds_base_kernel<<<blocks_for(out.w, out.h, block), block, 0, stream>>>(posts, col0, row0, pw,
                                                                          ph, out);
    return cudaGetLastError();
}

// The 2 x 2 blocks anchored at even coordinates that hold the nodes [lo, lo + n).
void block_range(int64_t lo, uint32_t n, int64_t& b0, uint32_t& count) {
    const auto half = [](int64_t v) { return v >= 0 ? v / 2 : -((1 - v) / 2); };
    b0 = half(lo);
    count = n == 0 ? 0u : uint32_t(half(lo + int64_t(n) - 1) - b0 + 1);
}

cudaError_t launch_ds_level(const DsLevel& parents, const DsLevel& out, int64_t c0, int64_t r0,
                            uint32_t w, uint32_t h, int level, double squareStep,
                            double diamondStep, uint32_t seed, bool spline,
                            cudaStream_t stream) {
    const dim3 block(32, 8);
    int64_t sc0, sr0, dc0, dr0;
    uint32_t sw, sh, dw, dh;
    block_range(out.c0, out.w, sc0, sw);
    block_range(out.r0, out.h, sr0, sh);
    block_range(c0, w, dc0, dw);
    block_range(r0, h, dr0, dh);
    if (spline) {
        ds_square_kernel<true><<<blocks_for(sw, sh, block), block, 0, stream>>>(
            parents, out, sc0, sr0, sw, sh, level, squareStep, seed);
        ds_diamond_kernel<true><<<blocks_for(dw, dh, block), block, 0, stream>>>(
            out, c0, r0, w, h, dc0, dr0, dw, dh, level, diamondStep, seed);
    } else {
        ds_square_kernel<false><<<blocks_for(sw, sh, block), block, 0, stream>>>(
            parents, out, sc0, sr0, sw, sh, level, squareStep, seed);
        ds_diamond_kernel<false><<<blocks_for(dw, dh, block), block, 0, stream>>>(
            out, c0, r0, w, h, dc0, dr0, dw, dh, level, diamondStep, seed);
    }
    return cudaGetLastError();
}

cudaError_t launch_ds_read(const DsLevel& nodes, const DsFrame& frame, const Grid& grid,
                           float* heights, cudaStream_t stream) {
    const dim3 block(32, 8);
    ds_read_kernel<<<blocks_for(grid.width, grid.height, block), block, 0, stream>>>(
        nodes, frame, grid, heights);
    return cudaGetLastError();
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
