// Diamond-square refinement of one output block in shared memory (Refinement::Refine and
// Interpolate, src/sources/diamond_square.cpp:426-485), shared by the plain refinement
// (diamond_square.cu: posts from an array) and the batch engine (batch.cu: posts from the source
// at the post lattice). Included by units compiled with -fmad=false, so the means and the read-out
// round as the reference's.
#pragma once

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
        // Each 32 x 32 -> 64-bit product in one wide multiply: its high and low words.
        const uint64_t p0 = uint64_t(0xD2511F53u) * c.x, p1 = uint64_t(0xCD9E8D57u) * c.z;
        c = Words{uint32_t(p1 >> 32) ^ c.y ^ k0, uint32_t(p1), uint32_t(p0 >> 32) ^ c.w ^ k1,
                  uint32_t(p0)};
    }
    return c;
}

// ln 2 split for k ln 2 + log1p(f) (Cody and Waite): the high part has 12 significant bits, so
// its product with any |k| <= 64 is exact in float.
constexpr float kLn2High = 0.693145751953125f;
constexpr float kLn2Low = float(0.69314718055994530942 - 0.693145751953125);
// pi 2^-52: a 53-bit integer times this is pi times the integer's share of 2^52.
constexpr float kPiOver2p52 = float(3.14159265358979323846 / 4503599627370496.0);

// log(n 2^-53) in float for an integer 1 <= n <= 2^53, with relative accuracy near n = 2^53
// (where the logarithm goes to 0), one path for every lane. n 2^-53 = 2^k (1 + f) with 1 + f in
// [0.75, 1.5) (f an integer difference, exact before its one rounding to float), and
// log(1 + f) = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + s^7/7 + s^9/9 + ...) for s = f / (2 + f),
// |s| <= 1/5, the series cut after s^9 (its tail is below 1e-8 of the sum): within 3e-7 of the
// logarithm relative.
__device__ __forceinline__ float log_of_ratio(uint64_t n) {
    const int bits = 64 - __clzll(n);  // n in [2^(bits - 1), 2^bits)
    const bool upper = n >= (3ull << (bits - 2 < 0 ? 0 : bits - 2)) && bits >= 2;
    const int e = upper ? bits : bits - 1;  // 1 + f = n / 2^e
    const float f = float(int64_t(n) - int64_t(1ull << e)) * __int_as_float((127 - e) << 23);
    const float s = __fdividef(f, 2.0f + f);
    const float s2 = s * s;
    float series = fmaf(s2, 1.0f / 9.0f, 1.0f / 7.0f);
    series = fmaf(s2, series, 1.0f / 5.0f);
    series = fmaf(s2, series, 1.0f / 3.0f);
    const float log1p = fmaf(2.0f * s * s2, series, 2.0f * s);
    const float k = float(e - 53);
    return fmaf(k, kLn2High, fmaf(k, kLn2Low, log1p));
}

// The standard normal of node (col, row) of `level` (Refinement::Displacement,
// diamond_square.cpp:382-389): one Philox block is RandomStream's first two NextDouble draws
// (u1, u2, 53 bits each, exact), turned into a normal by Box-Muller (StandardNormal,
// src/random/samplers.cpp:65-69), sqrt(-2 log(1 - u1)) cos(2 pi u2). The reference evaluates it
// in double; here in float on arguments formed exactly from the draws' integers: the logarithm
// as above, the square root as x rsqrt(x), and the cosine of pi a with a = 2 u2 moved into
// [-1, 1) by an exact integer subtraction (the hardware cosine is within 4e-7 there). Within 1e-5
// of the double normal (a few 1e-7 of the radius; under 2e-5 m in the refined heights), for the
// fewest instructions: the refinement is bound by issuing them.
__device__ __forceinline__ double node_normal(int64_t col, int64_t row, int level,
                                              uint32_t seed) {
    const uint32_t high = uint32_t((col >> 32) ^ (row >> 32));
    const Words b = philox(Words{uint32_t(col), uint32_t(row), uint32_t(level) | (high << 5), 0u},
                           seed, kMidpointDisplacementStream);
    // u1 = m1 2^-53 and u2 = m2 2^-53; 1 - u1 = (2^53 - m1) 2^-53 exactly.
    const uint64_t m1 = (uint64_t(b.x >> 5u) << 26u) | uint64_t(b.y >> 6u);
    const uint64_t m2 = (uint64_t(b.z >> 5u) << 26u) | uint64_t(b.w >> 6u);
    const float twice = -2.0f * log_of_ratio((1ull << 53) - m1);
    const float radius = twice > 0.0f ? twice * rsqrtf(twice) : 0.0f;
    // 2 u2 = m2 2^-52 in [0, 2), as m2 - 2^53 2^-52 in [-1, 0) from 1 on.
    const int64_t turn = int64_t(m2) - (m2 >= (1ull << 52) ? int64_t(1ull << 53) : int64_t(0));
    const float c = __cosf(float(turn) * kPiOver2p52);
    return double(radius * c);
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

// The threads that refine one block together: the whole CTA (a grid block), or one warp (a
// point, whose node boxes are a few nodes wide).
struct CtaGroup {
    __device__ __forceinline__ int32_t rank() const { return int32_t(threadIdx.x); }
    __device__ __forceinline__ int32_t size() const { return int32_t(blockDim.x); }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct WarpGroup {
    __device__ __forceinline__ int32_t rank() const { return int32_t(threadIdx.x & 31u); }
    __device__ __forceinline__ int32_t size() const { return 32; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
};

// Walks a w x h box (w > 0) in row-major order with a group's threads, thread k taking items k,
// k + n, k + 2n, ... (n threads): consecutive threads take neighbouring nodes, the work splits
// evenly, and a thread steps its (x, y) without dividing.
struct BoxWalk {
    int32_t x, y, dx, dy, w;
    template <class Group>
    __device__ __forceinline__ BoxWalk(int32_t width, const Group& g) : w(width) {
        const int32_t k = g.rank(), n = g.size();
        x = k % w;
        y = k / w;
        dx = n % w;
        dy = n / w;
    }
    __device__ __forceinline__ void next() {
        x += dx;
        y += dy;
        if (x >= w) {
            x -= w;
            ++y;
        }
    }
};

constexpr uint32_t kDsMaxBlock = 64;  // the largest block side the host picks

// Per-block shared state besides the node buffers.
struct DsShared {
    NodeBox inner[kMaxDsLevels + 1];
    int32_t colNode[kDsMaxBlock], rowNode[kDsMaxBlock];  // north-up grids: a column's and a row's
    double colShare[kDsMaxBlock], rowShare[kDsMaxBlock];  // finest node and share (read step)
    int fits;
};

// Level-0 nodes from a window of the post lattice: node (col, row) is post (col, -row), the
// window held being the lattice's columns col0.. and rows row0.., reads past it repeating its
// edge (BaseNodes, diamond_square.cpp:311; PostIndex, src/sources/lattice.h:99).
struct PostsFromArray {
    const float* posts;
    int64_t col0, row0;
    uint32_t pw, ph;
    __device__ __forceinline__ double operator()(int64_t nodeCol, int64_t nodeRow) const {
        const int64_t col = nodeCol - col0, row = -nodeRow - row0;
        const int64_t pc = col < 0 ? 0 : (col >= int64_t(pw) ? int64_t(pw) - 1 : col);
        const int64_t pr = row < 0 ? 0 : (row >= int64_t(ph) ? int64_t(ph) - 1 : row);
        return double(posts[size_t(pr) * pw + size_t(pc)]);
    }
};

// One CTA refines the nodes an output block reads, every level in shared memory, and writes
// only the block's heights (Refinement::Refine, diamond_square.cpp:426-448, with the boxes worked
// out top-down as its recursion does). The block is t.blockW x t.blockH cells of t.grid, or, for a
// point job (t.points set), the one point `block` (written at heights[t.pointIndex[block]], or
// heights[block] without an index). Node values do not depend on the box they are computed in:
// displacements are keyed by (seed, node, level) through Philox4x32-10 and means are local, so
// neighbouring blocks agree on every node they share.
//   level 0   nodes from `posts` (a functor of the node's column and row);
//   level l   the square step over the box the diamond step reads (SquareStep, :392-407: kept
//             parents and displaced odd/odd nodes), then the diamond step over the box the next
//             level reads (DiamondStep, :410-424), in place;
//   read      each cell from the finest level.
// Levels of even and odd number alternate between two shared buffers of t.capEven and t.capOdd
// doubles. The group's first thread works out the boxes; one that would outgrow its buffer (the host sizes them
// from the block's extent, so never) sets flag 1 and the CTA writes nothing. Loops run over local
// 32-bit box coordinates; only the displacement's key takes the node's 64-bit index.
template <bool kSpline, class Posts, class Group = CtaGroup>
__device__ __forceinline__ void ds_block(const DsTile& t, uint32_t block, const Posts& posts,
                                         float* heights, double* pool, DsShared& sh,
                                         const Group group = Group()) {
    constexpr int64_t kReach = kSpline ? 3 : 1;   // the diamond mean's reach (Refine's `reach`)
    constexpr int64_t kBefore = kSpline ? 1 : 0;  // parents a square mean reads before its block
    constexpr int64_t kAfter = kSpline ? 2 : 1;   // and after it; the read's nodes after a cell
    const bool single = t.points != nullptr;
    uint32_t c0 = 0, r0 = 0, cw = 1, rh = 1;
    double pointX = 0.0, pointY = 0.0;
    if (single) {
        pointX = t.points[2 * size_t(block)];
        pointY = t.points[2 * size_t(block) + 1];
    } else {
        const uint32_t bx = block % t.blocksX, by = block / t.blocksX;
        c0 = bx * t.blockW;
        r0 = by * t.blockH;
        cw = min(t.blockW, t.grid.width - c0);
        rh = min(t.blockH, t.grid.height - r0);
    }
    // The center of the block's cell (c, r), or the point.
    auto center = [&](uint32_t c, uint32_t r, double& x, double& y) {
        if (single) {
            x = pointX;
            y = pointY;
        } else {
            cell_center(t.grid, c0 + c, r0 + r, x, y);
        }
    };
    const int levels = t.levels;
    const bool northUp = !single && t.grid.rowRotation == 0.0 && t.grid.colRotation == 0.0;
    if (group.rank() == 0) {
        double umin = INFINITY, umax = -INFINITY, vmin = INFINITY, vmax = -INFINITY;
        for (int k = 0; k < 4; ++k) {
            double x, y;
            center((k & 1) ? cw - 1 : 0, (k & 2) ? rh - 1 : 0, x, y);
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
        sh.inner[levels] = NodeBox{fc0, fr0, int32_t(fc1 - fc0 + 1), int32_t(fr1 - fr0 + 1)};
        for (int l = levels; l >= 1 && ok; --l) {
            const NodeBox& b = sh.inner[l];
            const int64_t oc0 = b.c0 - kReach, oc1 = b.c0 + b.w - 1 + kReach;
            const int64_t or0 = b.r0 - kReach, or1 = b.r0 + b.h - 1 + kReach;
            ok = (oc1 - oc0 + 1) * (or1 - or0 + 1) <= int64_t((l & 1) ? t.capOdd : t.capEven);
            const int64_t pc0 = floor_half(oc0) - kBefore, pc1 = floor_half(oc1) + kAfter;
            const int64_t pr0 = floor_half(or0) - kBefore, pr1 = floor_half(or1) + kAfter;
            sh.inner[l - 1] = NodeBox{pc0, pr0, int32_t(pc1 - pc0 + 1), int32_t(pr1 - pr0 + 1)};
        }
        ok = ok && int64_t(sh.inner[0].w) * sh.inner[0].h <= int64_t(t.capEven);
        sh.fits = ok ? 1 : 0;
        if (!ok) {
            atomicOr(t.status, 1u);
        }
    }
    group.sync();
    if (!sh.fits) {
        return;
    }
    if (northUp) {
        // A north-up cell's x depends on its column alone and its y on its row alone (the other
        // term of cell_center is an exact zero), so their finest node (relative to the finest
        // box) and share are found once per column and row.
        const int64_t fc0 = sh.inner[levels].c0 - (levels > 0 ? kReach : 0);
        const int64_t fr0 = sh.inner[levels].r0 - (levels > 0 ? kReach : 0);
        for (uint32_t i = uint32_t(group.rank()); i < cw + rh; i += uint32_t(group.size())) {
            double x, y;
            int64_t node;
            double share;
            if (i < cw) {
                center(i, 0, x, y);
                node_and_share((x - t.frame.originX) / t.frame.stepX, node, share);
                sh.colShare[i] = share;
                sh.colNode[i] = int32_t(node - fc0);
            } else {
                center(0, i - cw, x, y);
                node_and_share((y - t.frame.originY) / t.frame.stepY, node, share);
                sh.rowShare[i - cw] = share;
                sh.rowNode[i - cw] = int32_t(node - fr0);
            }
        }
    }
    {
        const NodeBox p = sh.inner[0];
        for (BoxWalk it(p.w, group); it.y < p.h; it.next()) {
            pool[it.y * p.w + it.x] = posts(p.c0 + it.x, p.r0 + it.y);
        }
    }
    group.sync();
    NodeBox pb = sh.inner[0];
    const double* parents = pool;
    for (int l = 1; l <= levels; ++l) {
        const NodeBox d = sh.inner[l];
        const NodeBox ob{d.c0 - kReach, d.r0 - kReach, int32_t(d.w + 2 * kReach),
                         int32_t(d.h + 2 * kReach)};
        double* out = (l & 1) ? pool + t.capEven : pool;
        const double squareStep = t.squareStep[l], diamondStep = t.diamondStep[l];
        // Square step: the 2 x 2 blocks anchored at even (col, row) that meet the box. Block
        // (i, j) is parent (sc0 + i, sr0 + j); its even node sits at local (oc, orow) of the
        // output box and its odd/odd node one further along both axes. A thread takes two
        // neighbouring blocks of a row at a time and draws both displacements before it reads
        // any node, so their two Philox chains run interleaved.
        {
            const int64_t sc0 = floor_half(ob.c0), sr0 = floor_half(ob.r0);
            const int32_t sw = int32_t(floor_half(ob.c0 + ob.w - 1) - sc0 + 1);
            const int32_t shh = int32_t(floor_half(ob.r0 + ob.h - 1) - sr0 + 1);
            const int32_t pcBase = int32_t(sc0 - pb.c0), prBase = int32_t(sr0 - pb.r0);
            const int32_t ocBase = int32_t(2 * sc0 - ob.c0), orBase = int32_t(2 * sr0 - ob.r0);
            for (BoxWalk it((sw + 1) / 2, group); it.y < shh; it.next()) {
                const int32_t j = it.y;
                const int64_t row = 2 * (sr0 + j) + 1;
                double normal[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    normal[k] = node_normal(2 * (sc0 + 2 * it.x + k) + 1, row, l, t.seed);
                }
                const int32_t orow = orBase + 2 * j;
                const double* p0 = parents + (prBase + j) * pb.w + pcBase;
                const double* p1 = p0 + pb.w;
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int32_t i = 2 * it.x + k;
                    const int32_t oc = ocBase + 2 * i;
                    if (i >= sw) {
                        break;
                    }
                    if (oc >= 0 && orow >= 0) {
                        out[orow * ob.w + oc] = p0[i];
                    }
                    if (oc + 1 >= ob.w || orow + 1 >= ob.h) {
                        continue;
                    }
                    double mean;
                    if (!kSpline) {
                        mean = 0.25 * (p0[i] + p0[i + 1] + p1[i] + p1[i + 1]);
                    } else {
                        mean = 0.0;
                        for (int32_t b = 0; b < 4; ++b) {
                            const double* line = p0 + (b - 1) * pb.w + i - 1;
                            double acc = 0.0;
                            for (int32_t a = 0; a < 4; ++a) {
                                acc += kMid[a] * line[a];
                            }
                            mean += kMid[b] * acc;
                        }
                    }
                    out[(orow + 1) * ob.w + oc + 1] = mean + squareStep * normal[k];
                }
            }
        }
        group.sync();
        // Diamond step: the mixed nodes (2 bc + 1, 2 br) and (2 bc, 2 br + 1) inside the box the
        // next level reads, from the square step's nodes around them (kReach local columns and
        // rows of the output box lie before the inner box). Both displacements of a block are
        // drawn before its nodes are read.
        {
            const int64_t dc0 = floor_half(d.c0), dr0 = floor_half(d.r0);
            const int32_t dw = int32_t(floor_half(d.c0 + d.w - 1) - dc0 + 1);
            const int32_t dh = int32_t(floor_half(d.r0 + d.h - 1) - dr0 + 1);
            const int32_t lcBase = int32_t(2 * dc0 - d.c0), lrBase = int32_t(2 * dr0 - d.r0);
            for (BoxWalk it(dw, group); it.y < dh; it.next()) {
                const int32_t i = it.x, j = it.y;
                double normal[2];
#pragma unroll
                for (int n = 0; n < 2; ++n) {
                    // Inner-box local position of the node: (2 i + 1, 2 j) or (2 i, 2 j + 1).
                    const int32_t lc = lcBase + 2 * i + (n == 0 ? 1 : 0);
                    const int32_t lr = lrBase + 2 * j + (n == 0 ? 0 : 1);
                    normal[n] = node_normal(d.c0 + lc, d.r0 + lr, l, t.seed);
                }
#pragma unroll
                for (int n = 0; n < 2; ++n) {
                    const int32_t lc = lcBase + 2 * i + (n == 0 ? 1 : 0);
                    const int32_t lr = lrBase + 2 * j + (n == 0 ? 0 : 1);
                    if (lc < 0 || lc >= d.w || lr < 0 || lr >= d.h) {
                        continue;
                    }
                    double* at = out + (lr + int32_t(kReach)) * ob.w + lc + int32_t(kReach);
                    double mean;
                    if (!kSpline) {
                        mean = 0.25 * (at[-1] + at[1] + at[-ob.w] + at[ob.w]);
                    } else {
                        double alongX = 0.0, alongY = 0.0;
                        for (int32_t k = 0; k < 4; ++k) {
                            alongX += kMid[k] * at[-3 + 2 * k];
                            alongY += kMid[k] * at[(-3 + 2 * k) * ob.w];
                        }
                        mean = 0.5 * (alongX + alongY);
                    }
                    *at = mean + diamondStep * normal[n];
                }
            }
        }
        group.sync();
        parents = out;
        pb = ob;
    }
    // The read: consecutive threads take consecutive cells of a row.
    const Nodes finest{pb, const_cast<double*>(parents)};
    for (BoxWalk it(int32_t(cw), group); it.y < int32_t(rh); it.next()) {
        const uint32_t c = uint32_t(it.x), r = uint32_t(it.y);
        double value;
        if (northUp && !kSpline) {
            const int32_t lc = sh.colNode[c], lr = sh.rowNode[r];
            const double u = sh.colShare[c], v = sh.rowShare[r];
            const double* at = parents + lr * pb.w + lc;
            value = at[0];
            if (u > 0.0) {
                value = value * (1.0 - u) + at[1] * u;
            }
            if (v > 0.0) {
                double above = at[pb.w];
                if (u > 0.0) {
                    above = above * (1.0 - u) + at[pb.w + 1] * u;
                }
                value = value * (1.0 - v) + above * v;
            }
        } else {
            double x, y;
            center(c, r, x, y);
            value = read_nodes<kSpline>(finest, t.frame, x, y);
        }
        if (single) {
            heights[t.pointIndex != nullptr ? t.pointIndex[block] : block] = float(value);
        } else {
            heights[size_t(r0 + r) * t.pitch + c0 + c] = float(value);
        }
    }
}

}  // namespace
}  // namespace tgb
