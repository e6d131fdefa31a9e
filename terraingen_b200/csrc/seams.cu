// The seam a source chain adds to a later source in an earlier one's gaps
// (detail::BuildSeamField, src/sources/seam_field.cpp:663-710; SourceChain::FillGridGaps,
// src/sources/source_chain.cpp:167-192), on the device.
//
// From the samples on the seam lattice (1 where the earlier source has data, earlier minus later
// where both do):
//   1. the band: posts with data within 3 posts of a gap keep their difference (NearGaps);
//   2. the chamfer distance from each post to the nearest post with data (DataDistances), in the
//      reference's own relaxation order: rows top down then bottom up, each row as a recurrence
//      along it, so every distance (and carried value) has the reference's float bits; values
//      beyond the reach are never read back, so they are dropped and each thread runs a short
//      window of the recurrence;
//   3a. Feather: gap posts within `width` take the carried difference faded by a smoothstep;
//   3b. Height / Slope: gap posts within the reach (3 decay lengths, away from the lattice's 3
//      border posts) are solved for (-Laplacian + 1/L^2) d = 0, or its square, with the band's
//      values fixed: conjugate gradients in FP64 preconditioned by a symmetric multigrid V-cycle
//      (damped Jacobi smoothing in FP32, the coarsest level's residual and sweeps in FP64) over
//      the unknowns compacted on each level. The reference solves the same system per connected
//      region with Gauss-Seidel smoothing; the converged field is the same.
// The field is read between posts by Catmull-Rom interpolation (SeamField::At) when a grid's
// gaps are filled from the later source.
//
// Built with -fmad=false: the distances and the interpolation round as the reference's
// -ffp-contract=off build does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "kernels.h"

using namespace tgb;
using namespace tgb::api;

namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr int kBandPosts = 3;     // seam_field.cpp:29
constexpr int kBorderPosts = 3;   // seam_field.cpp:32
constexpr int kSegment = 32;      // cells of a row a thread of the distance passes writes
constexpr int kMaxLevels = 8;
constexpr size_t kTileSharedBytes = 200 * 1024;  // a distance window's shared memory at most

// --- band and fixed values ---------------------------------------------------------------

__global__ void count_data_kernel(const uint8_t* __restrict__ data, size_t n,
                                  unsigned long long* __restrict__ count) {
    unsigned long long mine = 0;
    for (size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += size_t(gridDim.x) * blockDim.x) {
        mine += data[k] != 0 ? 1u : 0u;
    }
    for (int d = 16; d > 0; d >>= 1) {
        mine += __shfl_down_sync(0xffffffffu, mine, d);
    }
    if ((threadIdx.x & 31u) == 0 && mine > 0) {
        atomicAdd(count, mine);
    }
}

// NearGaps (seam_field.cpp:117): 1 where a post without data lies within `radius` columns...
__global__ void gaps_across_kernel(const uint8_t* __restrict__ data, uint32_t w, uint32_t h,
                                   int radius, uint8_t* __restrict__ across) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= size_t(w) * h) {
        return;
    }
    const int col = int(k % w);
    const size_t row0 = k - size_t(col);
    uint8_t any = 0;
    for (int c = max(0, col - radius); c <= min(int(w) - 1, col + radius); ++c) {
        any |= data[row0 + size_t(c)] == 0 ? 1 : 0;
    }
    across[k] = any;
}

// ... then of those within `radius` rows; the posts with data there hold their difference.
__global__ void band_kernel(const uint8_t* __restrict__ data, const float* __restrict__ difference,
                            const uint8_t* __restrict__ across, uint32_t w, uint32_t h,
                            int radius, float* __restrict__ field) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= size_t(w) * h) {
        return;
    }
    const int row = int(k / w);
    const size_t col = k % w;
    uint8_t near = 0;
    for (int r = max(0, row - radius); r <= min(int(h) - 1, row + radius); ++r) {
        near |= across[size_t(r) * w + col];
    }
    const float d = difference[k];
    field[k] = data[k] != 0 && near != 0 && !isnan(d) ? d : 0.0f;
}

// --- distances (DataDistances, seam_field.cpp:151) -----------------------------------------

struct DistanceRow {
    const uint8_t* data;
    const float* field;    // the carried value of a post with data (Feather)
    float* distance;       // forward pass output, backward pass input
    float* carried;        // optional, as distance
    float* distanceOut;    // backward pass output
    float* carriedOut;
    uint32_t w, h;
    float dx, dy, diagonal;
    float cap;       // distances above it are dropped (+inf): they are never read back
    int window;      // cells of recurrence before a thread's segment
};

// The forward pass over row `row`: each post without data relaxes from its left neighbor, then
// the posts above, up-left and up-right (strictly smaller wins, in that order), the row above
// already final. Each thread writes kSegment posts, running the recurrence along the row from
// `window` posts before them.
__global__ void distance_forward_kernel(const DistanceRow p, uint32_t row) {
    const int c0 = int(blockIdx.x * blockDim.x + threadIdx.x) * kSegment;
    if (c0 >= int(p.w)) {
        return;
    }
    const int w = int(p.w);
    const size_t base = size_t(row) * p.w;
    const float inf = INFINITY;
    float left = inf, leftCarried = 0.0f;
    const int end = min(w, c0 + kSegment);
    for (int c = max(0, c0 - p.window); c < end; ++c) {
        const size_t k = base + size_t(c);
        float d, carried = p.data[k] != 0 && p.carried != nullptr ? p.field[k] : 0.0f;
        if (p.data[k] != 0) {
            d = 0.0f;
        } else {
            d = inf;
            if (c > 0) {
                const float t = left + p.dx;
                if (t < d) {
                    d = t;
                    carried = leftCarried;
                }
            }
            if (row > 0) {
                const size_t up = k - p.w;
                float t = p.distance[up] + p.dy;
                if (t < d) {
                    d = t;
                    if (p.carried) carried = p.carried[up];
                }
                if (c > 0) {
                    t = p.distance[up - 1] + p.diagonal;
                    if (t < d) {
                        d = t;
                        if (p.carried) carried = p.carried[up - 1];
                    }
                }
                if (c + 1 < w) {
                    t = p.distance[up + 1] + p.diagonal;
                    if (t < d) {
                        d = t;
                        if (p.carried) carried = p.carried[up + 1];
                    }
                }
            }
            if (d > p.cap) {
                d = inf;
            }
        }
        if (c >= c0) {
            p.distance[k] = d;
            if (p.carried) {
                p.carried[k] = carried;
            }
        }
        left = d;
        leftCarried = carried;
    }
}

// The backward pass over row `row`, right to left: a post without data keeps its forward value
// unless its right neighbor, then the posts below, down-right and down-left give a strictly
// smaller one. Forward values are read from `distance`, the rows below from `distanceOut`.
__global__ void distance_backward_kernel(const DistanceRow p, uint32_t row) {
    const int w = int(p.w);
    const int segment = int(blockIdx.x * blockDim.x + threadIdx.x);
    const int hi = w - 1 - segment * kSegment;  // this thread writes [lo, hi]
    if (hi < 0) {
        return;
    }
    const int lo = max(0, hi - kSegment + 1);
    const size_t base = size_t(row) * p.w;
    const float inf = INFINITY;
    float right = inf, rightCarried = 0.0f;
    for (int c = min(w - 1, hi + p.window); c >= lo; --c) {
        const size_t k = base + size_t(c);
        float d = p.distance[k];
        float carried = p.carried != nullptr ? p.carried[k] : 0.0f;
        if (p.data[k] == 0) {
            if (c + 1 < w) {
                const float t = right + p.dx;
                if (t < d) {
                    d = t;
                    carried = rightCarried;
                }
            }
            if (row + 1 < p.h) {
                const size_t down = k + p.w;
                float t = p.distanceOut[down] + p.dy;
                if (t < d) {
                    d = t;
                    if (p.carried) carried = p.carriedOut[down];
                }
                if (c + 1 < w) {
                    t = p.distanceOut[down + 1] + p.diagonal;
                    if (t < d) {
                        d = t;
                        if (p.carried) carried = p.carriedOut[down + 1];
                    }
                }
                if (c > 0) {
                    t = p.distanceOut[down - 1] + p.diagonal;
                    if (t < d) {
                        d = t;
                        if (p.carried) carried = p.carriedOut[down - 1];
                    }
                }
            }
            if (d > p.cap) {
                d = inf;
            }
        }
        if (c <= hi) {
            p.distanceOut[k] = d;
            if (p.carried) {
                p.carriedOut[k] = carried;
            }
        }
        right = d;
        rightCarried = carried;
    }
}

// --- distances by tiles ---------------------------------------------------------------------
//
// A distance at most `cap` comes from a path of steps that each add at least dx (a step across
// columns) or dy (across rows), so it reaches no further than cap / dx columns and cap / dy rows:
// both passes, run over a window that holds a tile plus a halo of mx = cap / dx + 2 columns and
// my = cap / dy + 2 rows (clipped to the lattice, whose edges the reference's passes start from
// too) and started from no distance outside it, give every post of the tile the reference's
// distance and carried value wherever the distance is at most `cap`. Larger values are never
// read back, so they are written as +inf. Inside a window the passes run as wavefronts: the
// forward pass reads the left, upper-left, upper and upper-right posts, all on earlier fronts
// 2 row + col, and the backward pass mirrors it, so every post sees the same operands, in the
// same order, as in the row-by-row relaxation.
//
// Only tiles that hold a post without data and see a post with data within their halo are
// computed; distance_init_kernel gives every other post its value (0 with data, +inf without).

struct DistanceTiles {
    const uint8_t* data;
    const float* field;  // the carried value of a post with data, or null (no carried values)
    float* distance;
    float* carried;
    uint32_t w, h;
    float dx, dy, diagonal, cap;
    int ts;              // tile side
    int mx, my;          // halo columns and rows
    int maxPosts;        // posts of the largest window
    uint32_t tilesX, tilesY;
    const uint32_t* list;
    const uint32_t* count;
};

__global__ void distance_init_kernel(const uint8_t* __restrict__ data,
                                     const float* __restrict__ field, size_t n,
                                     float* __restrict__ distance, float* __restrict__ carried) {
    for (size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n;
         k += size_t(gridDim.x) * blockDim.x) {
        const bool has = data[k] != 0;
        distance[k] = has ? 0.0f : INFINITY;
        if (carried != nullptr) {
            carried[k] = has ? field[k] : 0.0f;
        }
    }
}

// Posts with data per tile (one block per tile).
__global__ void tile_counts_kernel(const uint8_t* __restrict__ data, uint32_t w, uint32_t h,
                                   int ts, uint32_t tilesX, uint32_t* __restrict__ counts) {
    const uint32_t tile = blockIdx.x;
    const uint32_t r0 = (tile / tilesX) * uint32_t(ts), c0 = (tile % tilesX) * uint32_t(ts);
    const uint32_t rows = min(uint32_t(ts), h - r0), cols = min(uint32_t(ts), w - c0);
    uint32_t mine = 0;
    for (uint32_t i = threadIdx.x; i < rows * cols; i += blockDim.x) {
        mine += data[size_t(r0 + i / cols) * w + c0 + i % cols] != 0 ? 1u : 0u;
    }
    for (int d = 16; d > 0; d >>= 1) {
        mine += __shfl_down_sync(0xffffffffu, mine, d);
    }
    __shared__ uint32_t warps[32];
    if ((threadIdx.x & 31u) == 0) {
        warps[threadIdx.x >> 5] = mine;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t total = 0;
        for (uint32_t i = 0; i < (blockDim.x + 31) / 32; ++i) {
            total += warps[i];
        }
        counts[tile] = total;
    }
}

// The tiles to compute: a post without data, and a post with data within `rx` tiles across and
// `ry` down or up (a superset of the halo).
__global__ void active_tiles_kernel(const uint32_t* __restrict__ counts, uint32_t w, uint32_t h,
                                    int ts, uint32_t tilesX, uint32_t tilesY, int rx, int ry,
                                    uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
    const uint32_t tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= tilesX * tilesY) {
        return;
    }
    const int tx = int(tile % tilesX), ty = int(tile / tilesX);
    const uint32_t rows = min(uint32_t(ts), h - uint32_t(ty) * ts);
    const uint32_t cols = min(uint32_t(ts), w - uint32_t(tx) * ts);
    if (counts[tile] == rows * cols) {
        return;  // all posts have data
    }
    bool near = false;
    for (int y = max(0, ty - ry); y <= min(int(tilesY) - 1, ty + ry) && !near; ++y) {
        for (int x = max(0, tx - rx); x <= min(int(tilesX) - 1, tx + rx); ++x) {
            if (counts[size_t(y) * tilesX + x] != 0) {
                near = true;
                break;
            }
        }
    }
    if (near) {
        list[atomicAdd(count, 1u)] = tile;
    }
}

// Posts of the largest window of a tile of side `ts` on a w x h lattice, and the shared memory
// it takes.
size_t tile_window_posts(int ts, int mx, int my, uint32_t w, uint32_t h) {
    return std::min<size_t>(size_t(ts) + 2 * size_t(my), h) *
           std::min<size_t>(size_t(ts) + 2 * size_t(mx), w);
}

size_t tile_window_bytes(size_t posts, bool carried) {
    return posts * (carried ? 8 : 4) + ((posts + 31) / 32) * 4;
}

// One block per listed tile, blocks looping over the list.
__global__ void __launch_bounds__(128) distance_tile_kernel(const DistanceTiles p) {
    extern __shared__ float smem[];
    const uint32_t total = *p.count;
    const int maxPosts = p.maxPosts;
    float* F = smem;
    float* Cc = p.carried != nullptr ? smem + maxPosts : nullptr;
    uint32_t* bits = reinterpret_cast<uint32_t*>(smem + (p.carried != nullptr ? 2 : 1) * maxPosts);
    const int tid = int(threadIdx.x), lane = tid & 31, warp = tid >> 5, warps = blockDim.x >> 5;
    for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
        const uint32_t tile = p.list[item];
        const int r0 = int(tile / p.tilesX) * p.ts, c0 = int(tile % p.tilesX) * p.ts;
        const int rw0 = max(0, r0 - p.my), rw1 = min(int(p.h), r0 + p.ts + p.my);
        const int cw0 = max(0, c0 - p.mx), cw1 = min(int(p.w), c0 + p.ts + p.mx);
        const int hw = rw1 - rw0, ww = cw1 - cw0, posts = hw * ww;
        // Which window posts have data, one bit each.
        for (int base = warp * 32; base < posts; base += warps * 32) {
            const int i = base + lane;
            const bool has = i < posts &&
                             p.data[size_t(rw0 + i / ww) * p.w + size_t(cw0 + i % ww)] != 0;
            const uint32_t word = __ballot_sync(0xffffffffu, has);
            if (lane == 0) {
                bits[base >> 5] = word;
            }
        }
        __syncthreads();
        const int fronts = 2 * (hw - 1) + ww;
        // Forward: front t holds the posts with 2 row + col = t.
        for (int t = 0; t < fronts; ++t) {
            const int rlo = t >= ww ? (t - ww + 2) / 2 : 0, rhi = min(hw - 1, t / 2);
            for (int r = rlo + tid; r <= rhi; r += int(blockDim.x)) {
                const int c = t - 2 * r, k = r * ww + c;
                if ((bits[k >> 5] >> (k & 31)) & 1u) {
                    F[k] = 0.0f;
                    if (Cc) {
                        Cc[k] = p.field[size_t(rw0 + r) * p.w + size_t(cw0 + c)];
                    }
                    continue;
                }
                float d = INFINITY, carried = 0.0f;
                if (c > 0) {
                    const float s = F[k - 1] + p.dx;
                    if (s < d) {
                        d = s;
                        if (Cc) carried = Cc[k - 1];
                    }
                }
                if (r > 0) {
                    const int up = k - ww;
                    float s = F[up] + p.dy;
                    if (s < d) {
                        d = s;
                        if (Cc) carried = Cc[up];
                    }
                    if (c > 0) {
                        s = F[up - 1] + p.diagonal;
                        if (s < d) {
                            d = s;
                            if (Cc) carried = Cc[up - 1];
                        }
                    }
                    if (c + 1 < ww) {
                        s = F[up + 1] + p.diagonal;
                        if (s < d) {
                            d = s;
                            if (Cc) carried = Cc[up + 1];
                        }
                    }
                }
                F[k] = d;
                if (Cc) {
                    Cc[k] = carried;
                }
            }
            __syncthreads();
        }
        // Backward, in place: front t holds the posts with 2 (hw-1-row) + (ww-1-col) = t. A row
        // reads only the rows below it, so the pass stops at the tile's first row.
        const int hb = hw - (r0 - rw0);
        const int backFronts = 2 * (hb - 1) + ww;
        for (int t = 0; t < backFronts; ++t) {
            const int rlo = t >= ww ? (t - ww + 2) / 2 : 0, rhi = min(hb - 1, t / 2);
            for (int q = rlo + tid; q <= rhi; q += int(blockDim.x)) {
                const int r = hw - 1 - q, c = ww - 1 - (t - 2 * q), k = r * ww + c;
                if ((bits[k >> 5] >> (k & 31)) & 1u) {
                    continue;
                }
                float d = F[k];
                float carried = Cc ? Cc[k] : 0.0f;
                if (c + 1 < ww) {
                    const float s = F[k + 1] + p.dx;
                    if (s < d) {
                        d = s;
                        if (Cc) carried = Cc[k + 1];
                    }
                }
                if (r + 1 < hw) {
                    const int down = k + ww;
                    float s = F[down] + p.dy;
                    if (s < d) {
                        d = s;
                        if (Cc) carried = Cc[down];
                    }
                    if (c + 1 < ww) {
                        s = F[down + 1] + p.diagonal;
                        if (s < d) {
                            d = s;
                            if (Cc) carried = Cc[down + 1];
                        }
                    }
                    if (c > 0) {
                        s = F[down - 1] + p.diagonal;
                        if (s < d) {
                            d = s;
                            if (Cc) carried = Cc[down - 1];
                        }
                    }
                }
                F[k] = d;
                if (Cc) {
                    Cc[k] = carried;
                }
            }
            __syncthreads();
        }
        // The tile's posts without data.
        const int rows = min(p.ts, int(p.h) - r0), cols = min(p.ts, int(p.w) - c0);
        for (int i = tid; i < rows * cols; i += int(blockDim.x)) {
            const int r = r0 + i / cols - rw0, c = c0 + i % cols - cw0, k = r * ww + c;
            if ((bits[k >> 5] >> (k & 31)) & 1u) {
                continue;
            }
            const size_t g = size_t(rw0 + r) * p.w + size_t(cw0 + c);
            const float d = F[k];
            p.distance[g] = d <= p.cap ? d : INFINITY;
            if (Cc) {
                p.carried[g] = Cc[k];
            }
        }
        __syncthreads();
    }
}

// Feather (seam_field.cpp:218): gap posts within `width` take the carried difference, faded by a
// smoothstep from 1 at the edge to 0 at `width`.
__global__ void feather_kernel(const uint8_t* __restrict__ data,
                               const float* __restrict__ distance,
                               const float* __restrict__ carried, size_t n, double width,
                               float* __restrict__ field) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n || data[k] != 0 || !(distance[k] < width)) {
        return;
    }
    const double t = double(distance[k]) / width;
    const double weight = 1.0 - t * t * (3.0 - 2.0 * t);
    field[k] = float(weight * double(carried[k]));
}

// --- unknowns and the level hierarchy ------------------------------------------------------

// 1 at the posts solved for: no data, off the border, within the reach.
__global__ void unknown_kernel(const uint8_t* __restrict__ data,
                               const float* __restrict__ distance, uint32_t w, uint32_t h,
                               double reach, uint32_t* __restrict__ flags) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= size_t(w) * h) {
        return;
    }
    const uint32_t col = uint32_t(k % w), row = uint32_t(k / w);
    const bool inside = col >= uint32_t(kBorderPosts) && col + kBorderPosts < w &&
                        row >= uint32_t(kBorderPosts) && row + kBorderPosts < h;
    flags[k] = data[k] == 0 && inside && double(distance[k]) <= reach ? 1u : 0u;
}

// A coarser level's posts: the parents (col / 2, row / 2) of the finer level's unknowns.
__global__ void coarsen_kernel(const uint32_t* __restrict__ finePos, uint32_t n, uint32_t fineW,
                               uint32_t coarseW, uint32_t* __restrict__ coarseFlags) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) {
        return;
    }
    const uint32_t p = finePos[k];
    coarseFlags[size_t(p / fineW / 2) * coarseW + (p % fineW) / 2] = 1u;
}

// Flags (0 / 1) scanned in place into offsets: the compact index of each flagged post, its
// position, and ~0u at the others. `scanned` holds the exclusive scan, `flags` the marks.
__global__ void compact_kernel(const uint32_t* __restrict__ scanned,
                               const uint8_t* __restrict__ marks, size_t n,
                               uint32_t* __restrict__ index, uint32_t* __restrict__ position) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) {
        return;
    }
    if (marks[k] != 0) {
        position[scanned[k]] = uint32_t(k);
        index[k] = scanned[k];
    } else {
        index[k] = kNone;
    }
}

__global__ void flags_to_marks_kernel(const uint32_t* __restrict__ flags, size_t n,
                                      uint8_t* __restrict__ marks) {
    const size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) {
        marks[k] = flags[k] != 0 ? 1 : 0;
    }
}

// One level: its lattice, its unknowns and the operator's weights.
struct LevelView {
    uint32_t w, h, n;
    const uint32_t* index;     // [w * h] compact index or ~0u
    const uint32_t* position;  // [n] post of each unknown
    double cx, cy, center;     // 1/dx^2, 1/dy^2, 2 cx + 2 cy + 1/L^2
    double diagonal;           // the operator's center weight
    // Per unknown, the compact indices (or ~0u) of the posts the operator reads around it, in
    // kStencil order: 4 of them for order 1, 12 for order 2.
    const uint32_t* nbr;
    // Per unknown, the next coarser level's parent, across its column, across its row and
    // diagonally (Link, seam_field.cpp:367); null on the coarsest level.
    const uint32_t* parents;
    // Per unknown of a coarser level, the 4 x 4 finer posts (2C-1 .. 2C+2 by 2R-1 .. 2R+2) its
    // restriction gathers, row by row; null on the finest level.
    const uint32_t* children;
};

// The offsets of the 13-point stencil after its center (kNear13, seam_field.cpp:267); the first
// four are the 5-point stencil's.
__constant__ int2 kStencil[12] = {{-1, 0}, {1, 0},  {0, -1}, {0, 1},  {-2, 0}, {2, 0},
                                  {0, -2}, {0, 2},  {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};

// The operator at unknown k of u (0 off the unknowns): B = -Laplacian + 1/L^2 on 5 points
// (order 1), or B applied twice on 13 points (order 2), as ApplyScreened / Apply
// (seam_field.cpp:389-407), in the arithmetic of `A` (float on the FP32 levels).
template <typename T, typename A>
__device__ __forceinline__ A tap(const T* u, uint32_t j) {
    return j == kNone ? A(0) : A(u[j]);
}

template <int kOrder, typename T, typename A = double>
__device__ __forceinline__ A apply_at(const LevelView& L, const T* u, uint32_t k) {
    const uint4 n0 = reinterpret_cast<const uint4*>(L.nbr)[size_t(k) * (kOrder == 1 ? 1 : 3)];
    const A cx = A(L.cx), cy = A(L.cy), c0 = A(L.center);
    const A sx = tap<T, A>(u, n0.x) + tap<T, A>(u, n0.y);
    const A sy = tap<T, A>(u, n0.z) + tap<T, A>(u, n0.w);
    if (kOrder == 1) {
        return c0 * A(u[k]) - cx * sx - cy * sy;
    }
    const uint4 n1 = reinterpret_cast<const uint4*>(L.nbr)[size_t(k) * 3 + 1];
    const uint4 n2 = reinterpret_cast<const uint4*>(L.nbr)[size_t(k) * 3 + 2];
    const A s2x = tap<T, A>(u, n1.x) + tap<T, A>(u, n1.y);
    const A s2y = tap<T, A>(u, n1.z) + tap<T, A>(u, n1.w);
    const A sd = tap<T, A>(u, n2.x) + tap<T, A>(u, n2.y) + tap<T, A>(u, n2.z) +
                 tap<T, A>(u, n2.w);
    return A(L.diagonal) * A(u[k]) - A(2) * c0 * (cx * sx + cy * sy) + cx * cx * s2x +
           cy * cy * s2y + A(2) * cx * cy * sd;
}

// The stencil's neighbors of each unknown (compact indices, ~0u off the unknowns).
template <int kOrder>
__global__ void neighbors_kernel(const LevelView L, uint32_t* __restrict__ nbr) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= L.n) {
        return;
    }
    constexpr int kTaps = kOrder == 1 ? 4 : 12;
    const uint32_t p = L.position[k];
    const int col = int(p % L.w), row = int(p / L.w);
    for (int j = 0; j < kTaps; ++j) {
        const int c = col + kStencil[j].x, r = row + kStencil[j].y;
        nbr[size_t(k) * kTaps + j] =
            c < 0 || r < 0 || c >= int(L.w) || r >= int(L.h)
                ? kNone
                : L.index[size_t(r) * L.w + uint32_t(c)];
    }
}

// Each unknown's coarse parent and its neighbors across the unknown's column, row and diagonal.
__global__ void parents_kernel(const LevelView F, const LevelView Cl,
                               uint32_t* __restrict__ parents) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= F.n) {
        return;
    }
    const uint32_t p = F.position[k];
    const int col = int(p % F.w), row = int(p / F.w);
    const int pc = col / 2, pr = row / 2;
    const int ac = pc + (col % 2 == 1 ? 1 : -1), ar = pr + (row % 2 == 1 ? 1 : -1);
    const int cs[4] = {pc, ac, pc, ac}, rs[4] = {pr, pr, ar, ar};
    for (int j = 0; j < 4; ++j) {
        parents[size_t(k) * 4 + j] =
            cs[j] < 0 || rs[j] < 0 || cs[j] >= int(Cl.w) || rs[j] >= int(Cl.h)
                ? kNone
                : Cl.index[size_t(rs[j]) * Cl.w + uint32_t(cs[j])];
    }
}

// Each coarse unknown's 4 x 4 finer posts, as restriction gathers them.
__global__ void children_kernel(const LevelView F, const LevelView Cl,
                                uint32_t* __restrict__ children) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Cl.n) {
        return;
    }
    const uint32_t p = Cl.position[k];
    const int C = int(p % Cl.w), R = int(p / Cl.w);
    for (int j = 0; j < 4; ++j) {
        const int fy = 2 * R - 1 + j;
        for (int i = 0; i < 4; ++i) {
            const int fx = 2 * C - 1 + i;
            children[size_t(k) * 16 + j * 4 + i] =
                fx < 0 || fy < 0 || fx >= int(F.w) || fy >= int(F.h)
                    ? kNone
                    : F.index[size_t(fy) * F.w + uint32_t(fx)];
        }
    }
}

// The right-hand side: minus the operator of the fixed values (the field at every post that is
// not an unknown, 0 at the unknowns).
template <int kOrder>
__global__ void rhs_kernel(const LevelView L, const float* __restrict__ field,
                           double* __restrict__ rhs) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= L.n) {
        return;
    }
    const uint32_t p = L.position[k];
    const int col = int(p % L.w), row = int(p / L.w);
    auto f = [&](int dc, int dr) -> double {
        const size_t q = size_t(row + dr) * L.w + uint32_t(col + dc);
        return L.index[q] == kNone ? double(field[q]) : 0.0;
    };
    const double cx = L.cx, cy = L.cy, c0 = L.center;
    const double sx = f(-1, 0) + f(1, 0), sy = f(0, -1) + f(0, 1);
    double a;
    if (kOrder == 1) {
        a = -cx * sx - cy * sy;
    } else {
        const double s2x = f(-2, 0) + f(2, 0), s2y = f(0, -2) + f(0, 2);
        const double sd = f(-1, -1) + f(1, -1) + f(-1, 1) + f(1, 1);
        a = -2.0 * c0 * (cx * sx + cy * sy) + cx * cx * s2x + cy * cy * s2y + 2.0 * cx * cy * sd;
    }
    rhs[k] = -a;
}

// The conjugate gradients' scalars, on the device so an iteration needs no host round trip.
// Once `done` is set every kernel of an iteration returns at once, so iterations launched after
// the stop leave the solution as it was.
struct CgState {
    double fit;        // r . z of the current direction
    double target;     // the residual norm to stop at
    double step;
    double ratio;
    double dots[2];
    uint32_t done;
    uint32_t iterations;
    uint32_t maxIterations;
    uint32_t pad;
};

__device__ __forceinline__ bool stopped(const CgState* cg) {
    return cg != nullptr && cg->done != 0u;
}

// Damped Jacobi: xn = x + omega (b - A x) / diagonal; from x = 0 when `x` is null.
template <int kOrder, typename T>
__global__ void jacobi_kernel(const LevelView L, const T* __restrict__ b, const T* __restrict__ x,
                              T* __restrict__ xn, double omega, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= L.n || stopped(cg)) {
        return;
    }
    const T scale = T(omega / L.diagonal);
    if (x == nullptr) {
        xn[k] = scale * b[k];
        return;
    }
    const T r = b[k] - apply_at<kOrder, T, T>(L, x, k);
    xn[k] = x[k] + scale * r;
}

template <int kOrder, typename T>
__global__ void residual_kernel(const LevelView L, const T* __restrict__ b,
                                const T* __restrict__ x, T* __restrict__ r, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < L.n && !stopped(cg)) {
        r[k] = b[k] - apply_at<kOrder, T, T>(L, x, k);
    }
}

// The operator applied to a direction (FP64, for the conjugate gradients).
template <int kOrder>
__global__ void apply_kernel(const LevelView L, const double* __restrict__ u,
                             double* __restrict__ out, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < L.n && !stopped(cg)) {
        out[k] = apply_at<kOrder, double, double>(L, u, k);
    }
}

// Restriction, gathered: coarse unknown (C, R) takes 1/4 of each fine residual whose parent or
// parent's neighbor it is, weighted 3/4 or 1/4 per axis (the transfer weights 9/16, 3/16, 3/16,
// 1/16, seam_field.cpp:56).
template <typename Tf, typename Tc>
__global__ void restrict_kernel(const LevelView F, const LevelView Cl, const Tf* __restrict__ r,
                                Tc* __restrict__ b, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Cl.n || stopped(cg)) {
        return;
    }
    const double axis[4] = {0.25, 0.75, 0.75, 0.25};  // fine 2C-1, 2C, 2C+1, 2C+2
    const uint4* kids = reinterpret_cast<const uint4*>(Cl.children) + size_t(k) * 4;
    double sum = 0.0;
    for (int j = 0; j < 4; ++j) {
        const uint4 row = kids[j];
        const uint32_t q[4] = {row.x, row.y, row.z, row.w};
        for (int i = 0; i < 4; ++i) {
            if (q[i] != kNone) {
                sum += 0.25 * axis[i] * axis[j] * double(r[q[i]]);
            }
        }
    }
    b[k] = Tc(sum);
}

// Prolongation: each fine unknown adds its parent's correction and its parent's neighbors' across
// its column, its row and diagonally (Link, seam_field.cpp:367).
template <typename Tc, typename Tf>
__global__ void prolong_kernel(const LevelView F, const LevelView Cl, const Tc* __restrict__ xc,
                               Tf* __restrict__ x, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= F.n || stopped(cg)) {
        return;
    }
    const uint4 q = reinterpret_cast<const uint4*>(F.parents)[k];
    const double correction = 0.5625 * tap<Tc, double>(xc, q.x) +
                              0.1875 * tap<Tc, double>(xc, q.y) +
                              0.1875 * tap<Tc, double>(xc, q.z) +
                              0.0625 * tap<Tc, double>(xc, q.w);
    x[k] = Tf(double(x[k]) + correction);
}

// --- vectors -------------------------------------------------------------------------------

constexpr int kDotBlocks = 512;

// Partial sums of a . b (and of c . d when given) per block; summed by dot_finish_kernel in a
// fixed order, so every run gives the same bits.
__global__ void dot_kernel(const double* __restrict__ a, const double* __restrict__ b,
                           const double* __restrict__ c, const double* __restrict__ d, uint32_t n,
                           double* __restrict__ partial, const CgState* cg) {
    if (stopped(cg)) {
        return;
    }
    __shared__ double s0[256], s1[256];
    double x = 0.0, y = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        x += a[k] * b[k];
        if (c != nullptr) {
            y += c[k] * d[k];
        }
    }
    s0[threadIdx.x] = x;
    s1[threadIdx.x] = y;
    __syncthreads();
    for (int half = 128; half > 0; half >>= 1) {
        if (int(threadIdx.x) < half) {
            s0[threadIdx.x] += s0[threadIdx.x + half];
            s1[threadIdx.x] += s1[threadIdx.x + half];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = s0[0];
        partial[kDotBlocks + blockIdx.x] = s1[0];
    }
}

// The block partials summed by one block of kDotBlocks threads as a fixed tree, so every run
// adds them in the same order.
__global__ void dot_finish_kernel(const double* __restrict__ partial, double* __restrict__ out,
                                  const CgState* cg) {
    if (stopped(cg)) {
        return;
    }
    __shared__ double s0[kDotBlocks], s1[kDotBlocks];
    s0[threadIdx.x] = partial[threadIdx.x];
    s1[threadIdx.x] = partial[kDotBlocks + threadIdx.x];
    __syncthreads();
    for (int half = kDotBlocks / 2; half > 0; half >>= 1) {
        if (int(threadIdx.x) < half) {
            s0[threadIdx.x] += s0[threadIdx.x + half];
            s1[threadIdx.x] += s1[threadIdx.x + half];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s0[0];
        out[1] = s1[0];
    }
}

// After p . Ap: the step, or the stop when the curvature is not positive or the iterations are
// spent (PreconditionedCg, seam_field.cpp:519-527).
__global__ void cg_step_kernel(CgState* cg) {
    if (cg->done != 0u) {
        return;
    }
    const double curvature = cg->dots[0];
    if (cg->iterations >= cg->maxIterations || !(cg->fit > 0.0) || !(curvature > 0.0)) {
        cg->done = 1u;
        return;
    }
    cg->step = cg->fit / curvature;
    cg->iterations += 1u;
}

// After r . r and r . z: the stop at the target residual, else the direction's ratio
// (seam_field.cpp:532-542).
__global__ void cg_next_kernel(CgState* cg) {
    if (cg->done != 0u) {
        return;
    }
    if (sqrt(cg->dots[0]) <= cg->target) {
        cg->done = 1u;
        return;
    }
    const double next = cg->dots[1];
    cg->ratio = next / cg->fit;
    cg->fit = next;
}

// x += step p, r -= step ap.
__global__ void cg_update_kernel(double* __restrict__ x, double* __restrict__ r,
                                 const double* __restrict__ p, const double* __restrict__ ap,
                                 uint32_t n, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        const double step = cg->step;
        x[k] += step * p[k];
        r[k] -= step * ap[k];
    }
}

// p = z + ratio p.
__global__ void cg_direction_kernel(double* __restrict__ p, const double* __restrict__ z,
                                    uint32_t n, const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        p[k] = z[k] + cg->ratio * p[k];
    }
}

template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ in, B* __restrict__ out, uint32_t n,
                               const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        out[k] = B(in[k]);
    }
}

template <typename T>
__global__ void copy_kernel(const T* __restrict__ in, T* __restrict__ out, uint32_t n,
                            const CgState* cg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        out[k] = in[k];
    }
}

__global__ void scatter_solution_kernel(const uint32_t* __restrict__ position,
                                        const double* __restrict__ x, uint32_t n,
                                        float* __restrict__ field) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        field[position[k]] = float(x[k]);
    }
}

// --- reading the field (SeamField::At, seam_field.cpp:644) ---------------------------------

// The cubic convolution kernel (a = -0.5) of the reference's resampling (CubicWeight,
// src/raster/resample.cpp:20).
__device__ __forceinline__ double cubic_weight(double x) {
    const double a = -0.5;
    x = fabs(x);
    if (x <= 1.0) {
        return ((a + 2.0) * x - (a + 3.0)) * x * x + 1.0;
    }
    if (x < 2.0) {
        return ((a * x - 5.0 * a) * x + 8.0 * a) * x - 4.0 * a;
    }
    return 0.0;
}

struct SeamRead {
    const float* field;
    uint32_t w, h;          // the lattice
    double originX, pixelWidth, rowRotation, originY, colRotation, pixelHeight;
    bool set;               // any post set
    // Cells of the grid outside [c0, c1] x [r0, r1] read no post (a conservative box; the exact
    // test is seam_at's).
    int64_t c0, c1, r0, r1;
};

__device__ __forceinline__ double post(const SeamRead& s, double col, double row) {
    const long long c = (long long)col, r = (long long)row;
    if (c < 0 || r < 0 || c >= (long long)s.w || r >= (long long)s.h) {
        return 0.0;
    }
    return double(s.field[size_t(r) * s.w + size_t(c)]);
}

// The correction at (x, y): Catmull-Rom over the 4 x 4 posts around it, taps of zero weight
// skipped, as InterpolateLattice (src/raster/kernels.h:62) with ResampleMethod::Cubic.
__device__ double seam_at(const SeamRead& s, double x, double y) {
    if (!s.set) {
        return 0.0;
    }
    // GeoTransform::WorldToPixel (include/terraingen/raster/geo_transform.h:70)
    const double det = s.pixelWidth * s.pixelHeight - s.rowRotation * s.colRotation;
    const double dx = x - s.originX, dy = y - s.originY;
    const double px = (dx * s.pixelHeight - dy * s.rowRotation) / det;
    const double py = (dy * s.pixelWidth - dx * s.colRotation) / det;
    const double fx = px - 0.5, fy = py - 0.5;
    const double left = floor(fx), top = floor(fy);
    if (!(left >= -2.0 && top >= -2.0 && left <= double(s.w) && top <= double(s.h))) {
        return 0.0;
    }
    double wx[4], wy[4];
    for (int i = -1; i <= 2; ++i) {
        wx[i + 1] = cubic_weight((fx - left) - i);
        wy[i + 1] = cubic_weight((fy - top) - i);
    }
    double sum = 0.0;
    for (int j = -1; j <= 2; ++j) {
        for (int i = -1; i <= 2; ++i) {
            if (wx[i + 1] * wy[j + 1] == 0.0) {
                continue;
            }
            sum += wx[i + 1] * wy[j + 1] * post(s, left + i, top + j);
        }
    }
    return double(float(sum));
}

// FillGridGaps: each cell holding no data takes the later source's height plus the correction
// at its center (unchanged where the correction is 0; still no data where the later source has
// none).
// A cell is missing when it is not finite or, with a no-data value, equal to it
// (Raster::IsMissing, include/terraingen/raster/raster.h:167).
// Cells [c0, c0 + w) x [r0, r0 + h) of the grid, 4 adjacent cells of a row per thread.
struct FillWindow {
    uint32_t c0, r0, w, h;
};

__global__ void seam_fill_kernel(const SeamRead s, const Grid g, const FillWindow win,
                                 const float* __restrict__ later, const NoData nodata,
                                 float* __restrict__ heights) {
    const uint32_t first = (blockIdx.x * blockDim.x + threadIdx.x) * 4u;
    if (first >= win.w) {
        return;
    }
    for (uint32_t rr = blockIdx.y; rr < win.h; rr += gridDim.y) {
        const uint32_t row = win.r0 + rr;
        for (uint32_t j = first; j < min(first + 4u, win.w); ++j) {
            const uint32_t col = win.c0 + j;
            const size_t k = size_t(row) * g.width + col;
            const float cell = heights[k];
            const bool missing = !isfinite(cell) || (nodata.mode == 2u && cell == nodata.value);
            if (!missing) {
                continue;
            }
            const float value = later[k];
            const bool laterMissing =
                !isfinite(value) || (nodata.mode == 2u && value == nodata.value);
            if (laterMissing) {
                continue;
            }
            double correction = 0.0;
            if (int64_t(col) >= s.c0 && int64_t(col) <= s.c1 && int64_t(row) >= s.r0 &&
                int64_t(row) <= s.r1) {
                const double x = g.originX + (double(col) + 0.5) * g.pixelWidth +
                                 (double(row) + 0.5) * g.rowRotation;
                const double y = g.originY + (double(col) + 0.5) * g.colRotation +
                                 (double(row) + 0.5) * g.pixelHeight;
                correction = seam_at(s, x, y);
            }
            heights[k] = correction == 0.0 ? value : float(double(value) + correction);
        }
    }
}

// SampleSources on a window of a grid both sources are rasters on: post (i, j) is cell
// (col0 + i, row0 + j); off the grid neither source has data.
__global__ void seam_samples_kernel(const float* __restrict__ earlier,
                                    const float* __restrict__ later, uint32_t gw, uint32_t gh,
                                    int64_t col0, int64_t row0, uint32_t lw, uint32_t lh,
                                    const NoData nodata, uint8_t* __restrict__ data,
                                    float* __restrict__ difference) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lw) {
        return;
    }
    for (uint32_t j = blockIdx.y; j < lh; j += gridDim.y) {
        const int64_t col = col0 + int64_t(i), row = row0 + int64_t(j);
        const size_t k = size_t(j) * lw + i;
        uint8_t has = 0;
        float diff = NAN;
        if (col >= 0 && row >= 0 && col < int64_t(gw) && row < int64_t(gh)) {
            const size_t c = size_t(row) * gw + size_t(col);
            const float a = earlier[c];
            has = isfinite(a) && !(nodata.mode == 2u && a == nodata.value) ? 1 : 0;
            if (has) {
                const float b = later[c];
                if (isfinite(b) && !(nodata.mode == 2u && b == nodata.value)) {
                    diff = float(double(a) - double(b));
                }
            }
        }
        data[k] = has;
        difference[k] = diff;
    }
}

// Three timing events, released with the scope.
struct Events {
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    cudaError_t create() {
        for (cudaEvent_t& x : e) {
            if (cudaError_t err = cudaEventCreate(&x)) {
                return err;
            }
        }
        return cudaSuccess;
    }
    ~Events() {
        for (cudaEvent_t x : e) {
            if (x != nullptr) {
                cudaEventDestroy(x);
            }
        }
    }
};

uint32_t blocks_for(size_t n, uint32_t threads = 256) {
    return uint32_t((n + threads - 1) / threads);
}

// A level's device arrays.
struct Level {
    LevelView view{};
    Buffer index, position, x, b, t;  // x, b, t: float (double on the coarsest level)
    Buffer nbr, parents, children;
};

// The seam calls' device scratch, one per device, grown as needed and kept across calls (no
// allocation, and so no device-wide synchronization of a free, on a call that fits).
struct Work {
    Buffer marks, flags, scan, distance, carried, distance2, carried2, count, partial, dots;
    Buffer tileCounts, tileList, cg;
    Buffer cgX, cgR, cgP, cgAp, cgZ, rhs;
    Buffer hostIn, hostIn2, hostOut, hostOut2;  // device copies of host-memory arguments
    Level levels[kMaxLevels];
    ~Work() {
        for (Buffer* b : {&marks, &flags, &scan, &distance, &carried, &distance2, &carried2,
                          &count, &partial, &dots, &tileCounts, &tileList, &cg,
                          &cgX, &cgR, &cgP, &cgAp, &cgZ, &rhs,
                          &hostIn, &hostIn2, &hostOut, &hostOut2}) {
            b->release();
        }
        for (Level& l : levels) {
            for (Buffer* b : {&l.index, &l.position, &l.x, &l.b, &l.t, &l.nbr, &l.parents,
                              &l.children}) {
                b->release();
            }
        }
    }
};

Work& device_work(tg_device* d) {
    if (d->seams == nullptr) {
        d->seams = new Work();
        d->releaseSeams = [](void* w) { delete static_cast<Work*>(w); };
    }
    return *static_cast<Work*>(d->seams);
}

// Compacts `flags` (0 / 1 per post of a w x h lattice) into the level's index and positions.
int compact(Work& wk, Level& level, uint32_t w, uint32_t h, cudaStream_t s) {
    const size_t n = size_t(w) * h;
    if (n >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "a seam lattice holds fewer than 2^32 posts");
    }
    uint32_t* flags = static_cast<uint32_t*>(wk.flags.ptr);
    TG_CUDA(wk.marks.reserve(n), "allocation");
    flags_to_marks_kernel<<<blocks_for(n), 256, 0, s>>>(flags, n,
                                                       static_cast<uint8_t*>(wk.marks.ptr));
    TG_CUDA(wk.scan.reserve(scan_scratch_words(uint32_t(n)) * sizeof(uint32_t)), "allocation");
    TG_CUDA(launch_exclusive_scan(flags, uint32_t(n), static_cast<uint32_t*>(wk.scan.ptr), s),
            "scan");
    uint32_t total = 0;
    TG_CUDA(cudaMemcpyAsync(&total, flags + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy to host");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    TG_CUDA(level.index.reserve(n * sizeof(uint32_t)), "allocation");
    TG_CUDA(level.position.reserve(std::max<size_t>(total, 1) * sizeof(uint32_t)), "allocation");
    compact_kernel<<<blocks_for(n), 256, 0, s>>>(flags, static_cast<const uint8_t*>(wk.marks.ptr),
                                                n, static_cast<uint32_t*>(level.index.ptr),
                                                static_cast<uint32_t*>(level.position.ptr));
    TG_CUDA(cudaGetLastError(), "compact launch");
    level.view.w = w;
    level.view.h = h;
    level.view.n = total;
    level.view.index = static_cast<const uint32_t*>(level.index.ptr);
    level.view.position = static_cast<const uint32_t*>(level.position.ptr);
    return TG_OK;
}

struct Solver {
    Work* wk;
    int levels;
    int order;
    cudaStream_t s;
    double omega;
    int sweeps, coarsest;
    const CgState* cg;     // the device state iterations stop on (null: always run)
    cudaStream_t capture;  // a stream of the library's own, the iterations are captured on
};

double* cg_dots(CgState* cg) {
    return reinterpret_cast<double*>(reinterpret_cast<char*>(cg) + offsetof(CgState, dots));
}

template <int kOrder>
cudaError_t jacobi(const Solver& sv, const LevelView& L, const void* b, const void* x, void* xn,
                   bool coarsest) {
    if (coarsest) {
        jacobi_kernel<kOrder, double><<<blocks_for(L.n), 256, 0, sv.s>>>(
            L, static_cast<const double*>(b), static_cast<const double*>(x),
            static_cast<double*>(xn), sv.omega, sv.cg);
    } else {
        jacobi_kernel<kOrder, float><<<blocks_for(L.n), 256, 0, sv.s>>>(
            L, static_cast<const float*>(b), static_cast<const float*>(x),
            static_cast<float*>(xn), sv.omega, sv.cg);
    }
    return cudaGetLastError();
}

cudaError_t copy_level(const Solver& sv, const void* from, void* to, uint32_t n, bool wide) {
    if (wide) {
        copy_kernel<double><<<blocks_for(n), 256, 0, sv.s>>>(static_cast<const double*>(from),
                                                            static_cast<double*>(to), n, sv.cg);
    } else {
        copy_kernel<float><<<blocks_for(n), 256, 0, sv.s>>>(static_cast<const float*>(from),
                                                           static_cast<float*>(to), n, sv.cg);
    }
    return cudaGetLastError();
}

// The V-cycle from level `d` (VCycle, seam_field.cpp:423): an approximate solution of the level's
// operator for its b, from 0, into its x.
template <int kOrder>
int vcycle(Solver& sv, int d) {
    Level& L = sv.wk->levels[d];
    const bool last = d + 1 == sv.levels;
    if (L.view.n == 0) {
        return TG_OK;
    }
    const int sweeps = last ? sv.coarsest : sv.sweeps;
    // Sweeps alternate between x and t; the first starts from 0.
    void* cur = nullptr;
    for (int i = 0; i < sweeps; ++i) {
        void* next = (i % 2 == 0) ? L.x.ptr : L.t.ptr;
        TG_CUDA(jacobi<kOrder>(sv, L.view, L.b.ptr, cur, next, last), "jacobi");
        cur = next;
    }
    if (cur != L.x.ptr) {
        TG_CUDA(copy_level(sv, cur, L.x.ptr, L.view.n, last), "copy");
    }
    if (last) {
        return TG_OK;
    }
    Level& C = sv.wk->levels[d + 1];
    const bool coarseLast = d + 2 == sv.levels;
    // residual into t, restricted into the coarse b
    residual_kernel<kOrder, float><<<blocks_for(L.view.n), 256, 0, sv.s>>>(
        L.view, static_cast<const float*>(L.b.ptr), static_cast<const float*>(L.x.ptr),
        static_cast<float*>(L.t.ptr), sv.cg);
    if (coarseLast) {
        restrict_kernel<float, double><<<blocks_for(C.view.n), 256, 0, sv.s>>>(
            L.view, C.view, static_cast<const float*>(L.t.ptr), static_cast<double*>(C.b.ptr),
            sv.cg);
    } else {
        restrict_kernel<float, float><<<blocks_for(C.view.n), 256, 0, sv.s>>>(
            L.view, C.view, static_cast<const float*>(L.t.ptr), static_cast<float*>(C.b.ptr),
            sv.cg);
    }
    TG_CUDA(cudaGetLastError(), "restrict launch");
    if (int st = vcycle<kOrder>(sv, d + 1)) {
        return st;
    }
    if (coarseLast) {
        prolong_kernel<double, float><<<blocks_for(L.view.n), 256, 0, sv.s>>>(
            L.view, C.view, static_cast<const double*>(C.x.ptr), static_cast<float*>(L.x.ptr),
            sv.cg);
    } else {
        prolong_kernel<float, float><<<blocks_for(L.view.n), 256, 0, sv.s>>>(
            L.view, C.view, static_cast<const float*>(C.x.ptr), static_cast<float*>(L.x.ptr),
            sv.cg);
    }
    TG_CUDA(cudaGetLastError(), "prolong launch");
    for (int i = 0; i < sv.sweeps; ++i) {
        TG_CUDA(jacobi<kOrder>(sv, L.view, L.b.ptr, i % 2 == 0 ? L.x.ptr : L.t.ptr,
                               i % 2 == 0 ? L.t.ptr : L.x.ptr, false),
                "jacobi");
    }
    if (sv.sweeps % 2 == 1) {
        TG_CUDA(copy_level(sv, L.t.ptr, L.x.ptr, L.view.n, false), "copy");
    }
    return TG_OK;
}

// z = M r: the V-cycle on r (FP64 in, through FP32 levels, FP64 out).
template <int kOrder>
int precondition(Solver& sv, const double* r, double* z) {
    Level& L0 = sv.wk->levels[0];
    const uint32_t n = L0.view.n;
    if (sv.levels == 1) {
        TG_CUDA(copy_level(sv, r, L0.b.ptr, n, true), "copy");
        if (int st = vcycle<kOrder>(sv, 0)) {
            return st;
        }
        TG_CUDA(copy_level(sv, L0.x.ptr, z, n, true), "copy");
        return TG_OK;
    }
    convert_kernel<double, float><<<blocks_for(n), 256, 0, sv.s>>>(
        r, static_cast<float*>(L0.b.ptr), n, sv.cg);
    if (int st = vcycle<kOrder>(sv, 0)) {
        return st;
    }
    convert_kernel<float, double><<<blocks_for(n), 256, 0, sv.s>>>(
        static_cast<const float*>(L0.x.ptr), z, n, sv.cg);
    TG_CUDA(cudaGetLastError(), "convert launch");
    return TG_OK;
}

// a . b and c . d (c may be null) into `out` on the device.
cudaError_t dots(const Solver& sv, const double* a, const double* b, const double* c,
                 const double* d, uint32_t n, double* out) {
    dot_kernel<<<kDotBlocks, 256, 0, sv.s>>>(a, b, c, d, n,
                                             static_cast<double*>(sv.wk->partial.ptr), sv.cg);
    dot_finish_kernel<<<1, kDotBlocks, 0, sv.s>>>(static_cast<const double*>(sv.wk->partial.ptr),
                                                  out, sv.cg);
    return cudaGetLastError();
}

// Iterations launched between looks at whether the conjugate gradients stopped.
constexpr int kIterationsPerGraph = 4;

// One iteration of PreconditionedCg (seam_field.cpp:517-542), every scalar on the device.
template <int kOrder>
int iteration(Solver& sv, CgState* cg) {
    Work& wk = *sv.wk;
    const LevelView& L0 = wk.levels[0].view;
    const uint32_t n = L0.n;
    double* x = static_cast<double*>(wk.cgX.ptr);
    double* r = static_cast<double*>(wk.cgR.ptr);
    double* p = static_cast<double*>(wk.cgP.ptr);
    double* ap = static_cast<double*>(wk.cgAp.ptr);
    double* z = static_cast<double*>(wk.cgZ.ptr);
    apply_kernel<kOrder><<<blocks_for(n), 256, 0, sv.s>>>(L0, p, ap, cg);
    TG_CUDA(dots(sv, p, ap, nullptr, nullptr, n, cg_dots(cg)), "dot launch");
    cg_step_kernel<<<1, 1, 0, sv.s>>>(cg);
    cg_update_kernel<<<blocks_for(n), 256, 0, sv.s>>>(x, r, p, ap, n, cg);
    if (int st = precondition<kOrder>(sv, r, z)) {
        return st;
    }
    TG_CUDA(dots(sv, r, r, r, z, n, cg_dots(cg)), "dot launch");
    cg_next_kernel<<<1, 1, 0, sv.s>>>(cg);
    cg_direction_kernel<<<blocks_for(n), 256, 0, sv.s>>>(p, z, n, cg);
    TG_CUDA(cudaGetLastError(), "iteration launch");
    return TG_OK;
}

// PreconditionedCg (seam_field.cpp:497) on the finest level: the correction at the unknowns in
// cgX. The iterations run as a CUDA graph of kIterationsPerGraph of them, replayed until the
// device state says they stopped.
template <int kOrder>
int solve(Solver& sv, double tolerance, int maxIterations, int* iterations) {
    Work& wk = *sv.wk;
    const uint32_t n = wk.levels[0].view.n;
    double* x = static_cast<double*>(wk.cgX.ptr);
    double* r = static_cast<double*>(wk.cgR.ptr);
    double* p = static_cast<double*>(wk.cgP.ptr);
    CgState* cg = static_cast<CgState*>(wk.cg.ptr);
    TG_CUDA(cudaMemsetAsync(x, 0, size_t(n) * 8, sv.s), "memset");
    double* scratch = static_cast<double*>(wk.dots.ptr);
    sv.cg = nullptr;
    TG_CUDA(dots(sv, r, r, nullptr, nullptr, n, scratch), "dot launch");
    if (int st = precondition<kOrder>(sv, r, p)) {
        return st;
    }
    TG_CUDA(dots(sv, r, p, nullptr, nullptr, n, scratch + 2), "dot launch");
    double d[4];
    TG_CUDA(cudaMemcpyAsync(d, scratch, sizeof(d), cudaMemcpyDeviceToHost, sv.s), "copy");
    TG_CUDA(cudaStreamSynchronize(sv.s), "synchronize");
    CgState host{};
    host.fit = d[2];
    host.target = tolerance * std::sqrt(d[0]);
    host.maxIterations = uint32_t(maxIterations);
    host.done = host.fit > 0.0 ? 0u : 1u;
    *iterations = 0;
    if (host.done) {
        return TG_OK;
    }
    TG_CUDA(cudaMemcpyAsync(cg, &host, sizeof(host), cudaMemcpyHostToDevice, sv.s), "copy");
    TG_CUDA(cudaStreamSynchronize(sv.s), "synchronize");
    // Everything before is complete: the iterations run on the library's stream, which can be
    // captured whatever stream the caller gave.
    sv.cg = cg;
    sv.s = sv.capture;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    TG_CUDA(cudaStreamBeginCapture(sv.s, cudaStreamCaptureModeThreadLocal), "capture");
    int st = TG_OK;
    for (int i = 0; i < kIterationsPerGraph && st == TG_OK; ++i) {
        st = iteration<kOrder>(sv, cg);
    }
    const cudaError_t ended = cudaStreamEndCapture(sv.s, &graph);
    if (st != TG_OK || ended != cudaSuccess) {
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        return st != TG_OK ? st : fail(TG_ERROR_CUDA, "capture: %s", cudaGetErrorString(ended));
    }
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        return fail(TG_ERROR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    uint32_t state[2] = {0, 0};  // done, iterations
    for (int launched = 0; launched < maxIterations + kIterationsPerGraph;
         launched += kIterationsPerGraph) {
        e = cudaGraphLaunch(exec, sv.s);
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync(state, reinterpret_cast<char*>(cg) + offsetof(CgState, done),
                                sizeof(state), cudaMemcpyDeviceToHost, sv.s);
        }
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(sv.s);
        }
        if (e != cudaSuccess || state[0] != 0u) {
            break;
        }
    }
    cudaGraphExecDestroy(exec);
    if (e != cudaSuccess) {
        return fail(TG_ERROR_CUDA, "solve: %s", cudaGetErrorString(e));
    }
    *iterations = int(state[1]);
    return TG_OK;
}

thread_local tg_seam_stats g_last{};

}  // namespace

extern "C" {

int tg_seam_solve(tg_device* d, const uint8_t* data, const float* difference, uint32_t width,
                  uint32_t height, double dx, double dy, const tg_seam_options* options,
                  float* field, int memory, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    if (options == nullptr || data == nullptr || difference == nullptr || field == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "data, difference, options and field are required");
    }
    const tg_seam_options& o = *options;
    if (o.mode > 3u || !(dx > 0.0) || !(dy > 0.0) || !std::isfinite(dx) || !std::isfinite(dy) ||
        ((o.mode == 1u) && !(o.width > 0.0 && std::isfinite(o.width))) ||
        ((o.mode >= 2u) && !(o.decay_length > 0.0 && std::isfinite(o.decay_length))) ||
        o.levels < 1 || o.levels > kMaxLevels || o.sweeps < 1 || o.coarsest_sweeps < 1) {
        return fail(TG_ERROR_ARGUMENT, "seam options out of range");
    }
    const size_t n = size_t(width) * height;
    g_last = tg_seam_stats{};
    if (n == 0) {
        return TG_OK;
    }
    if (n >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "a seam lattice holds fewer than 2^32 posts");
    }
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    Work& wk = device_work(d);
    const uint8_t* dData = data;
    const float* dDiff = difference;
    float* dField = field;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(wk.hostIn.reserve(n), "allocation");
        TG_CUDA(wk.hostIn2.reserve(n * 4), "allocation");
        TG_CUDA(wk.hostOut.reserve(n * 4), "allocation");
        TG_CUDA(cudaMemcpyAsync(wk.hostIn.ptr, data, n, cudaMemcpyHostToDevice, s), "copy");
        TG_CUDA(cudaMemcpyAsync(wk.hostIn2.ptr, difference, n * 4, cudaMemcpyHostToDevice, s),
                "copy");
        dData = static_cast<const uint8_t*>(wk.hostIn.ptr);
        dDiff = static_cast<const float*>(wk.hostIn2.ptr);
        dField = static_cast<float*>(wk.hostOut.ptr);
    }
    // The call ends with its work done: the scratch it used is free for the next call, on
    // whatever stream that comes.
    auto finish = [&](int st) {
        if (st == TG_OK && memory == TG_MEMORY_HOST &&
            cudaMemcpyAsync(field, dField, n * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
            st = fail(TG_ERROR_CUDA, "copy to host");
        }
        const cudaError_t e = cudaStreamSynchronize(s);
        if (st == TG_OK && e != cudaSuccess) {
            st = fail(TG_ERROR_CUDA, "synchronize: %s", cudaGetErrorString(e));
        }
        return st;
    };
    TG_CUDA(cudaMemsetAsync(dField, 0, n * 4, s), "memset");
    Events ev;
    if (ev.create() != cudaSuccess) {
        return finish(fail(TG_ERROR_CUDA, "event"));
    }
    TG_CUDA(cudaEventRecord(ev.e[0], s), "event");
    if (o.mode == 0u) {
        return finish(TG_OK);
    }
    // The field is 0 when the earlier source has data at every post or at none.
    TG_CUDA(wk.count.reserve(8), "allocation");
    TG_CUDA(cudaMemsetAsync(wk.count.ptr, 0, 8, s), "memset");
    count_data_kernel<<<1184, 256, 0, s>>>(dData, n,
                                           static_cast<unsigned long long*>(wk.count.ptr));
    unsigned long long withData = 0;
    TG_CUDA(cudaMemcpyAsync(&withData, wk.count.ptr, 8, cudaMemcpyDeviceToHost, s), "copy");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    if (withData == 0 || withData == n) {
        return finish(TG_OK);
    }
    // The band's differences.
    TG_CUDA(wk.marks.reserve(n), "allocation");
    gaps_across_kernel<<<blocks_for(n), 256, 0, s>>>(dData, width, height, kBandPosts,
                                                    static_cast<uint8_t*>(wk.marks.ptr));
    band_kernel<<<blocks_for(n), 256, 0, s>>>(dData, dDiff, static_cast<uint8_t*>(wk.marks.ptr),
                                             width, height, kBandPosts, dField);
    TG_CUDA(cudaGetLastError(), "band launch");
    // Distances to the nearest post with data, up to the reach (Height, Slope) or the width
    // (Feather).
    const bool feather = o.mode == 1u;
    const double reach = feather ? o.width : 3.0 * o.decay_length;  // kSeamReachDecays
    TG_CUDA(wk.distance.reserve(n * 4), "allocation");
    if (feather) {
        TG_CUDA(wk.carried.reserve(n * 4), "allocation");
    }
    const float cap =
        float(reach) < reach ? std::nextafter(float(reach), INFINITY) : float(reach);
    const float* distance = nullptr;
    const float* carried = nullptr;
    // Halo of the tiled passes: a distance at most `cap` reaches cap / dx columns, cap / dy rows.
    const int mx = int(std::min(std::ceil(double(cap) / dx) + 2.0, double(width)));
    const int my = int(std::min(std::ceil(double(cap) / dy) + 2.0, double(height)));
    int ts = 0;
    for (int side : {128, 96, 64, 32}) {
        if (tile_window_bytes(tile_window_posts(side, mx, my, width, height), feather) <=
            kTileSharedBytes) {
            ts = side;
            break;
        }
    }
    if (ts > 0) {
        DistanceTiles t{};
        t.data = dData;
        t.field = feather ? dField : nullptr;
        t.distance = static_cast<float*>(wk.distance.ptr);
        t.carried = feather ? static_cast<float*>(wk.carried.ptr) : nullptr;
        t.w = width;
        t.h = height;
        t.dx = float(dx);
        t.dy = float(dy);
        t.diagonal = float(std::hypot(dx, dy));
        t.cap = cap;
        t.ts = ts;
        t.mx = mx;
        t.my = my;
        t.maxPosts = int(tile_window_posts(ts, mx, my, width, height));
        t.tilesX = (width + ts - 1) / ts;
        t.tilesY = (height + ts - 1) / ts;
        const size_t tiles = size_t(t.tilesX) * t.tilesY;
        TG_CUDA(wk.tileCounts.reserve(tiles * 4), "allocation");
        TG_CUDA(wk.tileList.reserve(tiles * 4 + 4), "allocation");
        uint32_t* counts = static_cast<uint32_t*>(wk.tileCounts.ptr);
        uint32_t* list = static_cast<uint32_t*>(wk.tileList.ptr);
        t.list = list + 1;
        t.count = list;
        distance_init_kernel<<<2368, 256, 0, s>>>(dData, dField, n, t.distance, t.carried);
        tile_counts_kernel<<<uint32_t(tiles), 256, 0, s>>>(dData, width, height, ts, t.tilesX,
                                                          counts);
        TG_CUDA(cudaMemsetAsync(list, 0, 4, s), "memset");
        active_tiles_kernel<<<blocks_for(tiles), 256, 0, s>>>(
            counts, width, height, ts, t.tilesX, t.tilesY, (mx + ts - 1) / ts,
            (my + ts - 1) / ts, list + 1, list);
        const size_t bytes = tile_window_bytes(size_t(t.maxPosts), feather);
        TG_CUDA(cudaFuncSetAttribute(distance_tile_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)),
                "shared memory attribute");
        int perSm = 0, sms = 0;
        TG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, distance_tile_kernel, 128,
                                                              bytes),
                "occupancy");
        TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->ordinal),
                "attribute");
        const uint32_t blocks = uint32_t(std::max(1, perSm) * sms);
        distance_tile_kernel<<<std::min<uint32_t>(blocks, uint32_t(tiles)), 128, bytes, s>>>(t);
        TG_CUDA(cudaGetLastError(), "distance launch");
        distance = t.distance;
        carried = t.carried;
    } else {
        // Halos too wide for a window in shared memory: the passes row by row.
        TG_CUDA(wk.distance2.reserve(n * 4), "allocation");
        if (feather) {
            TG_CUDA(wk.carried2.reserve(n * 4), "allocation");
        }
        DistanceRow row{};
        row.data = dData;
        row.field = dField;
        row.distance = static_cast<float*>(wk.distance.ptr);
        row.carried = feather ? static_cast<float*>(wk.carried.ptr) : nullptr;
        row.distanceOut = static_cast<float*>(wk.distance2.ptr);
        row.carriedOut = feather ? static_cast<float*>(wk.carried2.ptr) : nullptr;
        row.w = width;
        row.h = height;
        row.dx = float(dx);
        row.dy = float(dy);
        row.diagonal = float(std::hypot(dx, dy));
        row.cap = cap;
        // A recurrence along a row stays within the cap for at most cap / dx steps.
        row.window = mx;
        const uint32_t segments = (width + kSegment - 1) / kSegment;
        for (uint32_t r = 0; r < height; ++r) {
            distance_forward_kernel<<<blocks_for(segments, 128), 128, 0, s>>>(row, r);
        }
        for (uint32_t r = height; r-- > 0;) {
            distance_backward_kernel<<<blocks_for(segments, 128), 128, 0, s>>>(row, r);
        }
        TG_CUDA(cudaGetLastError(), "distance launch");
        distance = row.distanceOut;
        carried = row.carriedOut;
    }
    if (feather) {
        feather_kernel<<<blocks_for(n), 256, 0, s>>>(dData, distance, carried, n, o.width,
                                                    dField);
        TG_CUDA(cudaGetLastError(), "feather launch");
        return finish(TG_OK);
    }
    // The unknowns of each level.
    TG_CUDA(wk.flags.reserve((n + 1) * sizeof(uint32_t)), "allocation");
    unknown_kernel<<<blocks_for(n), 256, 0, s>>>(dData, distance, width, height, reach,
                                                static_cast<uint32_t*>(wk.flags.ptr));
    TG_CUDA(cudaGetLastError(), "unknown launch");
    const int order = o.mode == 3u ? 2 : 1;
    const double screening = 1.0 / (o.decay_length * o.decay_length);
    int levels = 0;
    uint32_t lw = width, lh = height;
    double ldx = dx, ldy = dy;
    for (; levels < int(o.levels); ++levels) {
        Level& L = wk.levels[levels];
        if (levels > 0) {
            const Level& F = wk.levels[levels - 1];
            lw = (lw + 1) / 2;
            lh = (lh + 1) / 2;
            ldx *= 2.0;
            ldy *= 2.0;
            TG_CUDA(cudaMemsetAsync(wk.flags.ptr, 0, (size_t(lw) * lh + 1) * sizeof(uint32_t), s),
                    "memset");
            coarsen_kernel<<<blocks_for(F.view.n), 256, 0, s>>>(
                F.view.position, F.view.n, F.view.w, lw, static_cast<uint32_t*>(wk.flags.ptr));
            TG_CUDA(cudaGetLastError(), "coarsen launch");
        }
        if (int st = compact(wk, L, lw, lh, s)) {
            return finish(st);
        }
        L.view.cx = 1.0 / (ldx * ldx);
        L.view.cy = 1.0 / (ldy * ldy);
        L.view.center = 2.0 * L.view.cx + 2.0 * L.view.cy + screening;
        L.view.diagonal = order == 1 ? L.view.center
                                     : L.view.center * L.view.center +
                                           2.0 * L.view.cx * L.view.cx +
                                           2.0 * L.view.cy * L.view.cy;
        if (levels == 0 && L.view.n == 0) {
            return finish(TG_OK);
        }
        if (L.view.n <= 32u || lw < 4 || lh < 4) {  // the coarsest, as kCoarsestPosts
            ++levels;
            break;
        }
    }
    for (int l = 0; l < levels; ++l) {
        Level& L = wk.levels[l];
        const size_t n1 = std::max<size_t>(L.view.n, 1);
        const size_t bytes = (l + 1 == levels ? 8 : 4) * n1;
        TG_CUDA(L.x.reserve(bytes), "allocation");
        TG_CUDA(L.b.reserve(bytes), "allocation");
        TG_CUDA(L.t.reserve(bytes), "allocation");
        // The operator's neighbors, and the links to the next coarser level both ways.
        const int taps = order == 1 ? 4 : 12;
        TG_CUDA(L.nbr.reserve(n1 * taps * 4), "allocation");
        L.view.nbr = static_cast<const uint32_t*>(L.nbr.ptr);
        if (L.view.n > 0) {
            if (order == 1) {
                neighbors_kernel<1><<<blocks_for(L.view.n), 256, 0, s>>>(
                    L.view, static_cast<uint32_t*>(L.nbr.ptr));
            } else {
                neighbors_kernel<2><<<blocks_for(L.view.n), 256, 0, s>>>(
                    L.view, static_cast<uint32_t*>(L.nbr.ptr));
            }
        }
        L.view.parents = nullptr;
        L.view.children = nullptr;
        if (l + 1 < levels) {
            Level& C = wk.levels[l + 1];
            TG_CUDA(L.parents.reserve(n1 * 16), "allocation");
            L.view.parents = static_cast<const uint32_t*>(L.parents.ptr);
            if (L.view.n > 0) {
                parents_kernel<<<blocks_for(L.view.n), 256, 0, s>>>(
                    L.view, C.view, static_cast<uint32_t*>(L.parents.ptr));
            }
        }
        if (l > 0) {
            const Level& F = wk.levels[l - 1];
            TG_CUDA(L.children.reserve(n1 * 64), "allocation");
            L.view.children = static_cast<const uint32_t*>(L.children.ptr);
            if (L.view.n > 0) {
                children_kernel<<<blocks_for(L.view.n), 256, 0, s>>>(
                    F.view, L.view, static_cast<uint32_t*>(L.children.ptr));
            }
        }
        TG_CUDA(cudaGetLastError(), "level links launch");
    }
    const uint32_t nu = wk.levels[0].view.n;
    for (Buffer* b : {&wk.cgX, &wk.cgR, &wk.cgP, &wk.cgAp, &wk.cgZ}) {
        TG_CUDA(b->reserve(size_t(nu) * 8), "allocation");
    }
    TG_CUDA(wk.partial.reserve(2 * kDotBlocks * 8), "allocation");
    TG_CUDA(wk.dots.reserve(32), "allocation");
    TG_CUDA(wk.cg.reserve(sizeof(CgState)), "allocation");
    TG_CUDA(cudaEventRecord(ev.e[1], s), "event");
    // The right-hand side from the fixed values, then the conjugate gradients.
    if (order == 1) {
        rhs_kernel<1><<<blocks_for(nu), 256, 0, s>>>(wk.levels[0].view, dField,
                                                    static_cast<double*>(wk.cgR.ptr));
    } else {
        rhs_kernel<2><<<blocks_for(nu), 256, 0, s>>>(wk.levels[0].view, dField,
                                                    static_cast<double*>(wk.cgR.ptr));
    }
    TG_CUDA(cudaGetLastError(), "rhs launch");
    Solver sv{&wk, levels, order, s, order == 1 ? 0.8 : 0.5, int(o.sweeps),
              int(o.coarsest_sweeps), nullptr, d->stream};
    int iterations = 0;
    const double tolerance = o.tolerance > 0.0 ? o.tolerance : 1e-10;
    const int st = order == 1 ? solve<1>(sv, tolerance, 200, &iterations)
                              : solve<2>(sv, tolerance, 200, &iterations);
    if (st != TG_OK) {
        return finish(st);
    }
    scatter_solution_kernel<<<blocks_for(nu), 256, 0, s>>>(
        wk.levels[0].view.position, static_cast<const double*>(wk.cgX.ptr), nu, dField);
    TG_CUDA(cudaGetLastError(), "scatter launch");
    TG_CUDA(cudaEventRecord(ev.e[2], s), "event");
    TG_CUDA(cudaEventSynchronize(ev.e[2]), "synchronize");
    float prepare = 0.0f, solved = 0.0f;
    cudaEventElapsedTime(&prepare, ev.e[0], ev.e[1]);
    cudaEventElapsedTime(&solved, ev.e[1], ev.e[2]);
    g_last.unknowns = nu;
    g_last.levels = uint32_t(levels);
    g_last.iterations = uint32_t(iterations);
    g_last.prepare_ms = prepare;
    g_last.solve_ms = solved;
    return finish(TG_OK);
}

int tg_seam_stats_get(tg_seam_stats* stats) {
    if (stats == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "stats is null");
    }
    *stats = g_last;
    return TG_OK;
}

int tg_seam_fill(tg_device* d, const float* field, const tg_grid* lattice, const float* later,
                 const tg_grid* grid, float* heights, tg_nodata nodata, const uint32_t* window,
                 int memory, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    Grid g, lg;
    if (int st = to_grid(grid, g)) {
        return st;
    }
    if (lattice == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "lattice is null");
    }
    lg = Grid{lattice->width,       lattice->height,       lattice->origin_x,
              lattice->pixel_width, lattice->row_rotation, lattice->origin_y,
              lattice->col_rotation, lattice->pixel_height};
    const double det = lg.pixelWidth * lg.pixelHeight - lg.rowRotation * lg.colRotation;
    if (!(det != 0.0) || !std::isfinite(det)) {
        return fail(TG_ERROR_ARGUMENT, "lattice transform must be invertible");
    }
    if (nodata.mode > 2u) {
        return fail(TG_ERROR_ARGUMENT, "nodata mode must be 0, 1 or 2");
    }
    const size_t cells = size_t(g.width) * g.height;
    const size_t posts = size_t(lg.width) * lg.height;
    if (cells == 0) {
        return TG_OK;
    }
    if (field == nullptr || later == nullptr || heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "field, later and heights are required");
    }
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    const float* df = field;
    const float* dl = later;
    float* dh = heights;
    auto done = [](int st) { return st; };
    if (memory == TG_MEMORY_HOST) {
        Work& wk = device_work(d);
        Buffer& bf = wk.hostIn2;
        Buffer& bl = wk.hostOut;
        Buffer& bh = wk.hostOut2;
        if (bf.reserve(std::max<size_t>(posts, 1) * 4) != cudaSuccess ||
            bl.reserve(cells * 4) != cudaSuccess || bh.reserve(cells * 4) != cudaSuccess) {
            return done(fail(TG_ERROR_MEMORY, "device allocation"));
        }
        if (cudaMemcpyAsync(bf.ptr, field, posts * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(bl.ptr, later, cells * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(bh.ptr, heights, cells * 4, cudaMemcpyHostToDevice, s) !=
                cudaSuccess) {
            return done(fail(TG_ERROR_CUDA, "copy to device"));
        }
        df = static_cast<const float*>(bf.ptr);
        dl = static_cast<const float*>(bl.ptr);
        dh = static_cast<float*>(bh.ptr);
    }
    // SeamField::At is 0 everywhere when no post was set; reading an all-zero field gives the
    // same 0, so the field is always read.
    const bool set = true;
    SeamRead sr{df,         lg.width,       lg.height,       lg.originX,
                lg.pixelWidth, lg.rowRotation, lg.originY,      lg.colRotation,
                lg.pixelHeight, set,           0,               int64_t(g.width) - 1,
                0,           int64_t(g.height) - 1};
    // Without rotations, the cells whose centers fall within 3 posts of the lattice: the field
    // reads no post anywhere else (SeamField::At's taps are the 4 x 4 posts around the point).
    if (lg.rowRotation == 0.0 && lg.colRotation == 0.0 && g.rowRotation == 0.0 &&
        g.colRotation == 0.0) {
        // Points whose lattice position is within [-3, n + 3] posts on both axes.
        const double xa = lg.originX - 3.0 * lg.pixelWidth;
        const double xb = lg.originX + (double(lg.width) + 3.0) * lg.pixelWidth;
        const double ya = lg.originY - 3.0 * lg.pixelHeight;
        const double yb = lg.originY + (double(lg.height) + 3.0) * lg.pixelHeight;
        const double xlo = std::min(xa, xb), xhi = std::max(xa, xb);
        const double ylo = std::min(ya, yb), yhi = std::max(ya, yb);
        // Cell (col, row) has its center at origin + (index + 0.5) * pixel.
        auto range = [](double lo, double hi, double origin, double pixel, int64_t n,
                        int64_t& a, int64_t& b) {
            double u = (lo - origin) / pixel - 0.5, v = (hi - origin) / pixel - 0.5;
            if (u > v) {
                std::swap(u, v);
            }
            if (!(std::isfinite(u) && std::isfinite(v))) {
                return;
            }
            u = std::clamp(u, -1e15, 1e15);
            v = std::clamp(v, -1e15, 1e15);
            a = std::max<int64_t>(0, int64_t(std::floor(u)) - 1);
            b = std::min<int64_t>(n - 1, int64_t(std::ceil(v)) + 1);
        };
        range(xlo, xhi, g.originX, g.pixelWidth, g.width, sr.c0, sr.c1);
        range(ylo, yhi, g.originY, g.pixelHeight, g.height, sr.r0, sr.r1);
    }
    const NoData nd{nodata.mode, nodata.value};
    FillWindow win{0, 0, g.width, g.height};
    if (window != nullptr) {
        win = FillWindow{window[0], window[1], window[2], window[3]};
        if (uint64_t(win.c0) + win.w > g.width || uint64_t(win.r0) + win.h > g.height) {
            return done(fail(TG_ERROR_ARGUMENT, "the fill window leaves the grid"));
        }
    }
    if (win.w > 0 && win.h > 0) {
        seam_fill_kernel<<<dim3(blocks_for((win.w + 3) / 4), std::min<uint32_t>(win.h, 65535u)),
                           256, 0, s>>>(sr, g, win, dl, nd, dh);
    }
    if (cudaGetLastError() != cudaSuccess) {
        return done(fail(TG_ERROR_CUDA, "seam fill launch"));
    }
    if (memory == TG_MEMORY_HOST) {
        if (cudaMemcpyAsync(heights, dh, cells * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            return done(fail(TG_ERROR_CUDA, "copy to host"));
        }
    }
    return done(TG_OK);
}

int tg_seam_samples(tg_device* d, const float* earlier, const float* later, const tg_grid* grid,
                    int64_t col0, int64_t row0, uint32_t lw, uint32_t lh, tg_nodata nodata,
                    uint8_t* data, float* difference, int memory, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    Grid g;
    if (int st = to_grid(grid, g)) {
        return st;
    }
    if (nodata.mode > 2u) {
        return fail(TG_ERROR_ARGUMENT, "nodata mode must be 0, 1 or 2");
    }
    const size_t posts = size_t(lw) * lh;
    const size_t cells = size_t(g.width) * g.height;
    if (posts == 0) {
        return TG_OK;
    }
    if (earlier == nullptr || later == nullptr || data == nullptr || difference == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "earlier, later, data and difference are required");
    }
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    auto done = [](int st) { return st; };
    const float* de = earlier;
    const float* dl = later;
    uint8_t* dd = data;
    float* df = difference;
    if (memory == TG_MEMORY_HOST) {
        Work& wk = device_work(d);
        Buffer& be = wk.hostIn2;
        Buffer& bl = wk.hostOut;
        Buffer& bd = wk.hostIn;
        Buffer& bf = wk.hostOut2;
        if (be.reserve(std::max<size_t>(cells, 1) * 4) != cudaSuccess ||
            bl.reserve(std::max<size_t>(cells, 1) * 4) != cudaSuccess ||
            bd.reserve(posts) != cudaSuccess || bf.reserve(posts * 4) != cudaSuccess) {
            return done(fail(TG_ERROR_MEMORY, "device allocation"));
        }
        if (cells > 0 &&
            (cudaMemcpyAsync(be.ptr, earlier, cells * 4, cudaMemcpyHostToDevice, s) !=
                 cudaSuccess ||
             cudaMemcpyAsync(bl.ptr, later, cells * 4, cudaMemcpyHostToDevice, s) !=
                 cudaSuccess)) {
            return done(fail(TG_ERROR_CUDA, "copy to device"));
        }
        de = static_cast<const float*>(be.ptr);
        dl = static_cast<const float*>(bl.ptr);
        dd = static_cast<uint8_t*>(bd.ptr);
        df = static_cast<float*>(bf.ptr);
    }
    seam_samples_kernel<<<dim3(blocks_for(lw), std::min<uint32_t>(lh, 65535u)), 256, 0, s>>>(
        de, dl, g.width, g.height, col0, row0, lw, lh, NoData{nodata.mode, nodata.value}, dd, df);
    if (cudaGetLastError() != cudaSuccess) {
        return done(fail(TG_ERROR_CUDA, "seam samples launch"));
    }
    if (memory == TG_MEMORY_HOST) {
        if (cudaMemcpyAsync(data, dd, posts, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(difference, df, posts * 4, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            return done(fail(TG_ERROR_CUDA, "copy to host"));
        }
    }
    return done(TG_OK);
}

}  // extern "C"
