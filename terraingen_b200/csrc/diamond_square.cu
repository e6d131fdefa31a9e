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

// Catmull-Rom weights of four nodes around a midpoint (diamond_square.cpp:37).
__device__ __constant__ const double kMid[4] = {-1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0, -1.0 / 16.0};

__device__ __forceinline__ int64_t floor_half(int64_t v) {  // FloorHalf, diamond_square.cpp:39
    return v >= 0 ? v / 2 : -((1 - v) / 2);
}

// A box of nodes [c0, c0 + w) x [r0, r0 + h) of one level, row-major in shared memory.
struct NodeBox {
    int64_t c0, r0;
    int32_t w, h;
};

struct Nodes {
    NodeBox b;
    double* v;
    __device__ __forceinline__ double at(int64_t col, int64_t row) const {
        return v[int32_t(row - b.r0) * b.w + int32_t(col - b.c0)];
    }
    __device__ __forceinline__ double& ref(int64_t col, int64_t row) const {
        return v[int32_t(row - b.r0) * b.w + int32_t(col - b.c0)];
    }
    __device__ __forceinline__ bool holds(int64_t col, int64_t row) const {
        return col >= b.c0 && col < b.c0 + b.w && row >= b.r0 && row < b.r0 + b.h;
    }
};

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

// The Keys cubic (a = -0.5) at an offset of `x` nodes (CubicWeight, src/raster/resample.cpp:20).
__device__ __forceinline__ double cubic_weight(double x) {
    x = fabs(x);
    if (x <= 1.0) {
        return (1.5 * x - 2.5) * x * x + 1.0;
    }
    if (x < 2.0) {
        return ((-0.5 * x + 2.5) * x - 4.0) * x + 2.0;
    }
    return 0.0;
}

// The finest nodes read at (x, y) (Refinement::Interpolate, diamond_square.cpp:461-485):
// bilinear, or Catmull-Rom over the 4 x 4 nodes around (InterpolateLatticeWeights with the
// cubic's KernelWeights, src/raster/kernels.h:32-51; taps of zero weight skipped).
template <bool kSpline>
__device__ __forceinline__ double read_nodes(const Nodes& n, const DsFrame& frame, double x,
                                             double y) {
    int64_t col, row;
    double u, v;
    node_and_share((x - frame.originX) / frame.stepX, col, u);
    node_and_share((y - frame.originY) / frame.stepY, row, v);
    if (kSpline) {
        double wx[4], wy[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            wx[i] = cubic_weight(u - double(i - 1));
            wy[i] = cubic_weight(v - double(i - 1));
        }
        double sum = 0.0;
        for (int j = 0; j < 4; ++j) {
            for (int i = 0; i < 4; ++i) {
                if (wx[i] * wy[j] == 0.0) {
                    continue;
                }
                sum += wx[i] * wy[j] * n.at(col - 1 + i, row - 1 + j);
            }
        }
        return sum;
    }
    double value = n.at(col, row);
    if (u > 0.0) {
        value = value * (1.0 - u) + n.at(col + 1, row) * u;
    }
    if (v > 0.0) {
        double above = n.at(col, row + 1);
        if (u > 0.0) {
            above = above * (1.0 - u) + n.at(col + 1, row + 1) * u;
        }
        value = value * (1.0 - v) + above * v;
    }
    return value;
}

__device__ __forceinline__ void cell_center(const Grid& g, uint32_t c, uint32_t r, double& x,
                                            double& y) {
    x = g.originX + (double(c) + 0.5) * g.pixelWidth + (double(r) + 0.5) * g.rowRotation;
    y = g.originY + (double(c) + 0.5) * g.colRotation + (double(r) + 0.5) * g.pixelHeight;
}

// One CTA refines the nodes an output block of `block` x `block` cells reads, every level in
// shared memory, and writes only the block's heights (Refinement::Refine, diamond_square.cpp:
// 426-448, with the boxes worked out top-down as its recursion does). Node values do not depend
// on the box they are computed in: displacements are keyed by (seed, node, level) through
// Philox4x32-10 and means are local, so neighbouring blocks agree on every node they share.
//   level 0   nodes from the posts: node (col, row) is post (col, -row) of the lattice, the
//             window held being its columns col0.. and rows row0.., reads past it repeating its
//             edge (BaseNodes, diamond_square.cpp:311; PostIndex, src/sources/lattice.h:99);
//   level l   the square step over the box the diamond step reads (SquareStep, :392-407: kept
//             parents and displaced odd/odd nodes), then the diamond step over the box the next
//             level reads (DiamondStep, :410-424), in place;
//   read      each cell from the finest level.
// Levels of even and odd number alternate between two shared buffers of t.capEven and t.capOdd
// doubles. Thread 0 works out the boxes; one that would outgrow its buffer (the host sizes them
// from the block's extent, so never) sets flag 1 and the CTA writes nothing.
template <bool kSpline>
__global__ void __launch_bounds__(kDsTileThreads) ds_tile_kernel(const DsTile t) {
    extern __shared__ double pool[];
    __shared__ NodeBox inner[kMaxDsLevels + 1];
    __shared__ int fits;
    constexpr int64_t kReach = kSpline ? 3 : 1;   // the diamond mean's reach (Refine's `reach`)
    constexpr int64_t kBefore = kSpline ? 1 : 0;  // parents a square mean reads before its block
    constexpr int64_t kAfter = kSpline ? 2 : 1;   // and after it; the read's nodes after a cell
    const uint32_t bx = blockIdx.x % t.blocksX, by = blockIdx.x / t.blocksX;
    const uint32_t c0 = bx * t.block, r0 = by * t.block;
    const uint32_t cw = min(t.block, t.grid.width - c0), rh = min(t.block, t.grid.height - r0);
    const int levels = t.levels;
    if (threadIdx.x == 0) {
        double umin = INFINITY, umax = -INFINITY, vmin = INFINITY, vmax = -INFINITY;
        for (int k = 0; k < 4; ++k) {
            double x, y;
            cell_center(t.grid, c0 + ((k & 1) ? cw - 1 : 0), r0 + ((k & 2) ? rh - 1 : 0), x, y);
            const double u = (x - t.frame.originX) / t.frame.stepX;
            const double v = (y - t.frame.originY) / t.frame.stepY;
            umin = fmin(umin, u);
            umax = fmax(umax, u);
            vmin = fmin(vmin, v);
            vmax = fmax(vmax, v);
        }
        const int64_t fc0 = int64_t(floor(umin)) - 1, fc1 = int64_t(ceil(umax)) + kAfter;
        const int64_t fr0 = int64_t(floor(vmin)) - 1, fr1 = int64_t(ceil(vmax)) + kAfter;
        bool ok = fc1 - fc0 < 65536 && fr1 - fr0 < 65536;
        inner[levels] = NodeBox{fc0, fr0, int32_t(fc1 - fc0 + 1), int32_t(fr1 - fr0 + 1)};
        for (int l = levels; l >= 1 && ok; --l) {
            const NodeBox& b = inner[l];
            const int64_t oc0 = b.c0 - kReach, oc1 = b.c0 + b.w - 1 + kReach;
            const int64_t or0 = b.r0 - kReach, or1 = b.r0 + b.h - 1 + kReach;
            ok = (oc1 - oc0 + 1) * (or1 - or0 + 1) <= int64_t((l & 1) ? t.capOdd : t.capEven);
            const int64_t pc0 = floor_half(oc0) - kBefore, pc1 = floor_half(oc1) + kAfter;
            const int64_t pr0 = floor_half(or0) - kBefore, pr1 = floor_half(or1) + kAfter;
            inner[l - 1] = NodeBox{pc0, pr0, int32_t(pc1 - pc0 + 1), int32_t(pr1 - pr0 + 1)};
        }
        ok = ok && int64_t(inner[0].w) * inner[0].h <= int64_t(t.capEven);
        fits = ok ? 1 : 0;
        if (!ok) {
            atomicOr(t.status, 1u);
        }
    }
    __syncthreads();
    if (!fits) {
        return;
    }
    Nodes parents{inner[0], pool};
    for (int32_t i = threadIdx.x; i < parents.b.w * parents.b.h; i += blockDim.x) {
        const int64_t col = parents.b.c0 + i % parents.b.w - t.col0;
        const int64_t row = -(parents.b.r0 + i / parents.b.w) - t.row0;
        const int64_t pc = col < 0 ? 0 : (col >= int64_t(t.pw) ? int64_t(t.pw) - 1 : col);
        const int64_t pr = row < 0 ? 0 : (row >= int64_t(t.ph) ? int64_t(t.ph) - 1 : row);
        parents.v[i] = double(t.posts[size_t(pr) * t.pw + size_t(pc)]);
    }
    __syncthreads();
    for (int l = 1; l <= levels; ++l) {
        const NodeBox& d = inner[l];
        const Nodes out{NodeBox{d.c0 - kReach, d.r0 - kReach, int32_t(d.w + 2 * kReach),
                                int32_t(d.h + 2 * kReach)},
                        (l & 1) ? pool + t.capEven : pool};
        // Square step: the 2 x 2 blocks anchored at even (col, row) that meet the box.
        const int64_t sc0 = floor_half(out.b.c0), sr0 = floor_half(out.b.r0);
        const int32_t sw = int32_t(floor_half(out.b.c0 + out.b.w - 1) - sc0 + 1);
        const int32_t sh = int32_t(floor_half(out.b.r0 + out.b.h - 1) - sr0 + 1);
        const double squareStep = t.squareStep[l], diamondStep = t.diamondStep[l];
        for (int32_t i = threadIdx.x; i < sw * sh; i += blockDim.x) {
            const int64_t bc = sc0 + i % sw, br = sr0 + i / sw;
            if (out.holds(2 * bc, 2 * br)) {
                out.ref(2 * bc, 2 * br) = parents.at(bc, br);
            }
            const int64_t col = 2 * bc + 1, row = 2 * br + 1;
            if (!out.holds(col, row)) {
                continue;
            }
            double mean;
            if (!kSpline) {
                mean = 0.25 * (parents.at(bc, br) + parents.at(bc + 1, br) +
                               parents.at(bc, br + 1) + parents.at(bc + 1, br + 1));
            } else {
                mean = 0.0;
                for (int64_t b = 0; b < 4; ++b) {
                    double line = 0.0;
                    for (int64_t a = 0; a < 4; ++a) {
                        line += kMid[a] * parents.at(bc - 1 + a, br - 1 + b);
                    }
                    mean += kMid[b] * line;
                }
            }
            out.ref(col, row) = mean + squareStep * node_normal(col, row, l, t.seed);
        }
        __syncthreads();
        // Diamond step: the mixed nodes (2 bc + 1, 2 br) and (2 bc, 2 br + 1) inside the box the
        // next level reads, from the square step's nodes around them.
        const int64_t dc0 = floor_half(d.c0), dr0 = floor_half(d.r0);
        const int32_t dw = int32_t(floor_half(d.c0 + d.w - 1) - dc0 + 1);
        const int32_t dh = int32_t(floor_half(d.r0 + d.h - 1) - dr0 + 1);
        const Nodes inside{d, nullptr};
        for (int32_t i = threadIdx.x; i < dw * dh; i += blockDim.x) {
            const int64_t bc = dc0 + i % dw, br = dr0 + i / dw;
            const int64_t cols[2] = {2 * bc + 1, 2 * bc}, rows[2] = {2 * br, 2 * br + 1};
#pragma unroll
            for (int n = 0; n < 2; ++n) {
                const int64_t col = cols[n], row = rows[n];
                if (!inside.holds(col, row)) {
                    continue;
                }
                double mean;
                if (!kSpline) {
                    mean = 0.25 * (out.at(col - 1, row) + out.at(col + 1, row) +
                                   out.at(col, row - 1) + out.at(col, row + 1));
                } else {
                    double alongX = 0.0, alongY = 0.0;
                    for (int64_t k = 0; k < 4; ++k) {
                        alongX += kMid[k] * out.at(col - 3 + 2 * k, row);
                        alongY += kMid[k] * out.at(col, row - 3 + 2 * k);
                    }
                    mean = 0.5 * (alongX + alongY);
                }
                out.ref(col, row) = mean + diamondStep * node_normal(col, row, l, t.seed);
            }
        }
        __syncthreads();
        parents = out;
    }
    // The read: consecutive threads take consecutive cells of a row.
    for (uint32_t i = threadIdx.x; i < cw * rh; i += blockDim.x) {
        const uint32_t c = c0 + i % cw, r = r0 + i / cw;
        double x, y;
        cell_center(t.grid, c, r, x, y);
        t.heights[size_t(r) * t.grid.width + c] = float(read_nodes<kSpline>(parents, t.frame, x, y));
    }
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


}  // namespace

cudaError_t launch_ds_tiles(const DsTile& t, bool spline, cudaStream_t stream) {
    const uint32_t blocks = t.blocksX * ((t.grid.height + t.block - 1) / t.block);
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
