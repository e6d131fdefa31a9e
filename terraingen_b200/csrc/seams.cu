// The seam a source chain adds to a later source in an earlier one's gaps
// (detail::BuildSeamField, src/sources/seam_field.cpp:663-710; SourceChain::FillGridGaps,
// src/sources/source_chain.cpp:167-192), on the device.
//
// From the samples on the seam lattice (1 where the earlier source has data, earlier minus later
// where both do):
//   1. the band: posts with data within 3 posts of a gap keep their difference (NearGaps);
//   2. the chamfer distance from each post to the nearest post with data (DataDistances), with
//      every post relaxed from the same neighbors in the same order as the reference's rows top
//      down then bottom up, so every distance (and carried value) has its float bits; values
//      beyond the reach are never read back, so each tile of the lattice is run in a window of
//      its own, one warp per tile;
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
#include <utility>
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
constexpr int kMaxLevels = 8;
constexpr size_t kRowSharedBytes = 200 * 1024;   // a distance block's rows in shared memory
constexpr size_t kScratchBytes = size_t(1) << 30;  // the distance warps' stored steps at most

// --- the band, in bits ------------------------------------------------------------------------
//
// The prepare passes keep the lattice's masks one bit per post: word j of row r holds columns
// 32 j .. 32 j + 31 (bit = column % 32), `pitch` = ceil(w / 32) words a row, the bits past the
// last column 0.

constexpr int kBandRows = 16;  // rows of a band warp's span

__device__ __forceinline__ uint32_t row_tail_mask(uint32_t j, uint32_t pitch, uint32_t w) {
    return j + 1 == pitch && (w & 31u) != 0 ? (1u << (w & 31u)) - 1u : 0xffffffffu;
}

// Which posts have data, one bit each, and how many have. A warp packs 8 words per pass, their
// 8 loads in flight together.
constexpr uint32_t kPackWords = 8;

__global__ void pack_data_kernel(const uint8_t* __restrict__ data, uint32_t w, uint32_t h,
                                 uint32_t pitch, uint32_t* __restrict__ bits,
                                 unsigned long long* __restrict__ count) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t words = pitch * h;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    uint32_t mine = 0;
    for (uint32_t q0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kPackWords; q0 < words;
         q0 += warps * kPackWords) {
        uint8_t v[kPackWords];
#pragma unroll
        for (uint32_t k = 0; k < kPackWords; ++k) {
            const uint32_t q = q0 + k;
            const uint32_t row = q / pitch, col = (q % pitch) * 32u + lane;
            v[k] = q < words && col < w ? data[size_t(row) * w + col] : uint8_t(0);
        }
#pragma unroll
        for (uint32_t k = 0; k < kPackWords; ++k) {
            const uint32_t word = __ballot_sync(0xffffffffu, v[k] != 0);
            if (lane == k && q0 + k < words) {
                bits[q0 + k] = word;
            }
            mine += __popc(word);
        }
    }
    if (lane == 0 && mine != 0) {
        atomicAdd(count, static_cast<unsigned long long>(mine));
    }
}

struct BandBits {
    const uint32_t* bits;
    const float* difference;
    float* field;
    uint32_t* tileCounts;  // posts with data per distance tile
    uint32_t w, h, pitch;
    int ts;
    uint32_t tilesX;
};

// NearGaps (seam_field.cpp:117) and the band's values: a post with data keeps its difference
// where a post without data lies within 3 columns and 3 rows of it; every other post is 0. A
// warp takes 32 words across (lane = word) and kBandRows rows down, dilating each row's gap bits
// by 3 columns with funnel shifts and OR-ing the last 7 rows as it goes; the field is written a
// row of 32 posts at a time. The posts with data are counted per distance tile on the way.
__global__ void band_bits_kernel(const BandBits p) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t spans = (p.pitch + 31u) / 32u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t j0 = (warp % spans) * 32u, j = j0 + lane;
    const int q0 = int(warp / spans) * kBandRows;
    if (q0 >= int(p.h)) {
        return;
    }
    const int q1 = min(int(p.h), q0 + kBandRows);
    const bool inWord = j < p.pitch;
    const uint32_t valid = inWord ? row_tail_mask(j, p.pitch, p.w) : 0u;
    auto word_at = [&](int q, uint32_t jj) -> uint32_t {
        return p.bits[size_t(q) * p.pitch + jj];
    };
    uint32_t near[7] = {0, 0, 0, 0, 0, 0, 0};  // dilated gaps of rows q-6 .. q
    uint32_t has[4] = {0, 0, 0, 0};             // data bits of rows q-3 .. q
    uint32_t counted = 0;
    int countRow = q0;
    for (int q = q0 - kBandPosts; q < q1 + kBandPosts; ++q) {
        const bool rowIn = q >= 0 && q < int(p.h);
        const uint32_t d = rowIn && inWord ? word_at(q, j) : 0u;
        const uint32_t g = rowIn ? ~d & valid : 0u;
        uint32_t gl = __shfl_up_sync(0xffffffffu, g, 1);
        uint32_t gr = __shfl_down_sync(0xffffffffu, g, 1);
        if (lane == 0) {
            gl = rowIn && j0 > 0 ? ~word_at(q, j0 - 1) : 0u;
        }
        if (lane == 31) {
            gr = rowIn && j + 1 < p.pitch ? ~word_at(q, j + 1) & row_tail_mask(j + 1, p.pitch, p.w)
                                          : 0u;
        }
        uint32_t dil = g;
#pragma unroll
        for (int s = 1; s <= kBandPosts; ++s) {
            dil |= __funnelshift_l(gl, g, s) | __funnelshift_r(g, gr, s);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            near[k] = near[k + 1];
        }
        near[6] = dil;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            has[k] = has[k + 1];
        }
        has[3] = d;
        const int c = q - kBandPosts;  // the row whose 7 rows of gaps are in
        if (c < q0) {
            continue;
        }
        const uint32_t band =
            has[0] & (near[0] | near[1] | near[2] | near[3] | near[4] | near[5] | near[6]);
        if (p.tileCounts != nullptr) {
            if (c / p.ts != countRow / p.ts) {
                if (counted != 0) {
                    atomicAdd(&p.tileCounts[uint32_t(countRow / p.ts) * p.tilesX + j * 32u / p.ts],
                              counted);
                }
                counted = 0;
                countRow = c;
            }
            counted += __popc(has[0]);
        }
        const size_t base = size_t(c) * p.w;
        for (int k = 0; k < 32; ++k) {
            const uint32_t b = __shfl_sync(0xffffffffu, band, k);
            const uint32_t col = (j0 + uint32_t(k)) * 32u + lane;
            if (col < p.w) {
                float v = 0.0f;
                if ((b >> lane) & 1u) {
                    v = p.difference[base + col];
                    v = isnan(v) ? 0.0f : v;
                }
                p.field[base + col] = v;
            }
        }
    }
    if (p.tileCounts != nullptr && counted != 0) {
        atomicAdd(&p.tileCounts[uint32_t(countRow / p.ts) * p.tilesX + j * 32u / p.ts], counted);
    }
}

// --- distances (DataDistances, seam_field.cpp:151) -----------------------------------------
//
// A distance at most `cap` comes from a path of steps that each add at least dx (a step across
// columns) or dy (across rows), so it reaches no further than cap / dx columns and cap / dy rows:
// both passes, run over a window that holds a tile plus a halo of mx = cap / dx + 2 columns and
// my = cap / dy + 2 rows (clipped to the lattice, whose edges the reference's passes start from
// too) and started from no distance outside it, give every post of the tile the reference's
// distance and carried value wherever the distance is at most `cap`; larger values are never
// read back. Only tiles that hold a post without data and see a post with data within their halo
// are computed.
//
// One warp runs a tile's window. The forward pass reads the left, upper-left, upper and
// upper-right posts: the warp takes the window's rows 32 at a time (lane = row), lane l at column
// t - 2 l on step t, so the row above has just passed the three columns a post reads, and they
// come across by shuffles (lane 0 reads the band above from a row in shared memory, which lane 31
// writes as it goes). The backward pass mirrors it from the bottom right, starting from the
// forward values, which the forward pass stores per step as 32 lanes (coalesced both ways: the
// backward step reads one stored step of the forward pass, lanes reversed). Every post sees the
// same operands in the same order as in the reference's row-by-row relaxation, so distances and
// carried values have its float bits. The backward pass stops at the tile's first row (a row
// reads only the rows below it). Each tile post's result goes straight out: its unknown bit
// (Height, Slope) or its Feather value.

struct DistanceWarps {
    const uint32_t* bits;  // data bits
    const float* field;    // the carried value of a post with data (Feather), or null
    uint32_t w, h, pitch;
    float dx, dy, diagonal;
    int ts;                // tile side, a multiple of 32
    int mx, my;            // halo columns and rows
    int rowFloats;         // floats of a warp's row in shared memory (or in `rows`)
    uint32_t tilesX;
    const uint32_t* list;
    const uint32_t* count;
    float* scratch;        // per warp slot: the forward pass's stored steps (then carried)
    size_t scratchFloats;  // per warp slot
    float* rows;           // per warp slot, when the rows are not in shared memory
    uint32_t slots;        // warps of the launch
    // Height / Slope: the unknowns (no data, 3 posts off the border, distance within `reach`).
    uint32_t* unknown;
    double reach;
    // Feather: gap posts within `width` take the carried difference faded by a smoothstep.
    float* feather;
    double width;
};

constexpr int kDistanceWarps = 4;  // warps of a distance block
constexpr int kGroup = 16;         // steps of a pass run between reads of their operands

template <bool kCarried, bool kSharedRows>
__global__ void __launch_bounds__(32 * kDistanceWarps)
    distance_warp_kernel(const DistanceWarps p) {
    extern __shared__ float smem[];
    const int lane = int(threadIdx.x & 31u), warp = int(threadIdx.x >> 5);
    const uint32_t slot = blockIdx.x * kDistanceWarps + uint32_t(warp);
    if (slot >= p.slots) {
        return;
    }
    float* rowF = kSharedRows ? smem + size_t(warp) * p.rowFloats * (kCarried ? 2 : 1)
                              : p.rows + size_t(slot) * p.rowFloats * (kCarried ? 2 : 1);
    float* rowC = rowF + p.rowFloats;
    float* store = p.scratch + size_t(slot) * p.scratchFloats;
    const float inf = INFINITY;
    const uint32_t total = *p.count;
    for (uint32_t item = slot; item < total; item += p.slots) {
        const uint32_t tile = p.list[item];
        const int r0 = int(tile / p.tilesX) * p.ts, c0 = int(tile % p.tilesX) * p.ts;
        const int rw0 = max(0, r0 - p.my), rw1 = min(int(p.h), r0 + p.ts + p.my);
        const int cw0 = max(0, c0 - p.mx), cw1 = min(int(p.w), c0 + p.ts + p.mx);
        const int ww = cw1 - cw0, steps = ww + 62;
        const int bandsAbove = (r0 - rw0 + 31) / 32, bandsBelow = (rw1 - r0 + 31) / 32;
        const int tr1 = min(int(p.h), r0 + p.ts), tc1 = min(int(p.w), c0 + p.ts);
        float* storeC = store + size_t(bandsBelow) * steps * 32;
        for (int c = lane; c < ww; c += 32) {
            rowF[c] = inf;
            if (kCarried) rowC[c] = 0.0f;
        }
        __syncwarp();
        // Forward, bands top down.
        for (int band = -bandsAbove; band < bandsBelow; ++band) {
            const int row = r0 + 32 * band + lane;
            const bool active = row >= rw0 && row < rw1;
            const size_t rowBits = size_t(active ? row : rw0) * p.pitch;
            float h1 = inf, h2 = inf, h3 = inf;
            float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
            uint32_t word = 0, next = 0;
            if (active) {
                word = p.bits[rowBits + uint32_t(cw0 >> 5)];
                next = (cw0 >> 5) + 1 < int(p.pitch) ? p.bits[rowBits + uint32_t(cw0 >> 5) + 1]
                                                     : 0u;
            }
            float* out = store + size_t(max(band, 0)) * steps * 32;
            float* outC = storeC + size_t(max(band, 0)) * steps * 32;
            for (int t0 = 0; t0 < steps; t0 += kGroup) {
            // Lane 0's row above over the group's columns t0 - 1 .. t0 + kGroup, read at once
            // (lane 31 of this band writes only columns left of them meanwhile).
            float above[kGroup + 2], aboveC[kGroup + 2];
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i < kGroup + 2; ++i) {
                    const int col = t0 - 1 + i;
                    const bool in = col >= 0 && col < ww;
                    above[i] = in ? rowF[col] : inf;
                    if (kCarried) aboveC[i] = in ? rowC[col] : 0.0f;
                }
            }
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                const int t = t0 + u;
                if (t >= steps) {
                    break;
                }
                const int c = t - 2 * lane;
                float uR = __shfl_up_sync(0xffffffffu, h1, 1);
                float uU = __shfl_up_sync(0xffffffffu, h2, 1);
                float uL = __shfl_up_sync(0xffffffffu, h3, 1);
                float vR = 0.0f, vU = 0.0f, vL = 0.0f;
                if (kCarried) {
                    vR = __shfl_up_sync(0xffffffffu, g1, 1);
                    vU = __shfl_up_sync(0xffffffffu, g2, 1);
                    vL = __shfl_up_sync(0xffffffffu, g3, 1);
                }
                if (lane == 0) {
                    uL = above[u];
                    uU = above[u + 1];
                    uR = above[u + 2];
                    if (kCarried) {
                        vL = aboveC[u];
                        vU = aboveC[u + 1];
                        vR = aboveC[u + 2];
                    }
                }
                float d = inf, car = 0.0f;
                if (active && c >= 0 && c < ww) {
                    const int x = cw0 + c;
                    if ((x & 31) == 0 && c > 0) {
                        word = next;
                        next = (x >> 5) + 1 < int(p.pitch) ? p.bits[rowBits + uint32_t(x >> 5) + 1]
                                                           : 0u;
                    }
                    if ((word >> (x & 31)) & 1u) {
                        d = 0.0f;
                        if (kCarried) car = p.field[size_t(row) * p.w + uint32_t(x)];
                    } else {
                        float s = h1 + p.dx;
                        if (s < d) {
                            d = s;
                            car = g1;
                        }
                        s = uU + p.dy;
                        if (s < d) {
                            d = s;
                            car = vU;
                        }
                        s = uL + p.diagonal;
                        if (s < d) {
                            d = s;
                            car = vL;
                        }
                        s = uR + p.diagonal;
                        if (s < d) {
                            d = s;
                            car = vR;
                        }
                    }
                    if (lane == 31) {
                        rowF[c] = d;
                        if (kCarried) rowC[c] = car;
                    }
                }
                h3 = h2;
                h2 = h1;
                h1 = d;
                if (kCarried) {
                    g3 = g2;
                    g2 = g1;
                    g1 = car;
                }
                if (band >= 0) {
                    out[size_t(t) * 32 + lane] = d;
                    if (kCarried) outC[size_t(t) * 32 + lane] = car;
                }
            }
            }
            __syncwarp();
        }
        // Backward, bands bottom up over the tile's rows and the halo below; lane 0 is a band's
        // lowest row.
        for (int c = lane; c < ww; c += 32) {
            rowF[c] = inf;
            if (kCarried) rowC[c] = 0.0f;
        }
        __syncwarp();
        for (int band = bandsBelow - 1; band >= 0; --band) {
            const int row = r0 + 32 * band + 31 - lane;
            const bool active = row < rw1;
            const size_t rowBits = size_t(active ? row : r0) * p.pitch;
            float h1 = inf, h2 = inf, h3 = inf;
            float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
            uint32_t word = 0, next = 0, unknownBits = 0;
            const int last = cw1 - 1;
            if (active) {
                word = p.bits[rowBits + uint32_t(last >> 5)];
                next = (last >> 5) > 0 ? p.bits[rowBits + uint32_t(last >> 5) - 1] : 0u;
            }
            const float* in = store + size_t(band) * steps * 32;
            const float* inC = storeC + size_t(band) * steps * 32;
            const bool tileRow = active && row < tr1;
            // The forward values of a group's steps are loaded a group ahead (they come from L2).
            float cur[kGroup], curC[kGroup];
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                const size_t at = size_t(ww + 61 - u) * 32 + uint32_t(31 - lane);
                cur[u] = u < steps ? in[at] : inf;
                if (kCarried) curC[u] = u < steps ? inC[at] : 0.0f;
            }
            for (int t0 = 0; t0 < steps; t0 += kGroup) {
            float nxt[kGroup], nxtC[kGroup];
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                const int t = t0 + kGroup + u;
                const size_t at = size_t(ww + 61 - t) * 32 + uint32_t(31 - lane);
                nxt[u] = t < steps ? in[at] : inf;
                if (kCarried) nxtC[u] = t < steps ? inC[at] : 0.0f;
            }
            // Lane 0's row below over the group's columns ww - t0 down to ww - t0 - kGroup - 1
            // (lane 31 writes only columns right of them meanwhile).
            float below[kGroup + 2], belowC[kGroup + 2];
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i < kGroup + 2; ++i) {
                    const int col = ww - t0 - i;
                    const bool ok = col >= 0 && col < ww;
                    below[i] = ok ? rowF[col] : inf;
                    if (kCarried) belowC[i] = ok ? rowC[col] : 0.0f;
                }
            }
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                const int t = t0 + u;
                if (t >= steps) {
                    break;
                }
                const int c = ww - 1 - t + 2 * lane;
                float dL = __shfl_up_sync(0xffffffffu, h1, 1);
                float dD = __shfl_up_sync(0xffffffffu, h2, 1);
                float dR = __shfl_up_sync(0xffffffffu, h3, 1);
                float eL = 0.0f, eD = 0.0f, eR = 0.0f;
                if (kCarried) {
                    eL = __shfl_up_sync(0xffffffffu, g1, 1);
                    eD = __shfl_up_sync(0xffffffffu, g2, 1);
                    eR = __shfl_up_sync(0xffffffffu, g3, 1);
                }
                if (lane == 0) {
                    dR = below[u];
                    dD = below[u + 1];
                    dL = below[u + 2];
                    if (kCarried) {
                        eR = belowC[u];
                        eD = belowC[u + 1];
                        eL = belowC[u + 2];
                    }
                }
                float d = inf, car = 0.0f;
                if (active && c >= 0 && c < ww) {
                    const int x = cw0 + c;
                    if ((x & 31) == 31 && c < ww - 1) {
                        word = next;
                        next = (x >> 5) > 0 ? p.bits[rowBits + uint32_t(x >> 5) - 1] : 0u;
                    }
                    d = cur[u];
                    if (kCarried) car = curC[u];
                    const bool has = (word >> (x & 31)) & 1u;
                    if (!has) {
                        float s = h1 + p.dx;
                        if (s < d) {
                            d = s;
                            car = g1;
                        }
                        s = dD + p.dy;
                        if (s < d) {
                            d = s;
                            car = eD;
                        }
                        s = dR + p.diagonal;
                        if (s < d) {
                            d = s;
                            car = eR;
                        }
                        s = dL + p.diagonal;
                        if (s < d) {
                            d = s;
                            car = eL;
                        }
                    }
                    if (lane == 31) {
                        rowF[c] = d;
                        if (kCarried) rowC[c] = car;
                    }
                    if (tileRow && x >= c0 && x < tc1) {
                        if (p.unknown != nullptr) {
                            const bool inside = x >= kBorderPosts && x + kBorderPosts < int(p.w) &&
                                                row >= kBorderPosts &&
                                                row + kBorderPosts < int(p.h);
                            if (!has && inside && double(d) <= p.reach) {
                                unknownBits |= 1u << (x & 31);
                            }
                            if ((x & 31) == 0) {
                                p.unknown[rowBits + uint32_t(x >> 5)] = unknownBits;
                                unknownBits = 0;
                            }
                        } else if (!has && double(d) < p.width) {
                            const double u = double(d) / p.width;
                            const double weight = 1.0 - u * u * (3.0 - 2.0 * u);
                            p.feather[size_t(row) * p.w + uint32_t(x)] =
                                float(weight * double(car));
                        }
                    }
                }
                h3 = h2;
                h2 = h1;
                h1 = d;
                if (kCarried) {
                    g3 = g2;
                    g2 = g1;
                    g1 = car;
                }
            }
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                cur[u] = nxt[u];
                if (kCarried) curC[u] = nxtC[u];
            }
            }
            __syncwarp();
        }
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

// --- unknowns and the level hierarchy ------------------------------------------------------
//
// A level's unknowns are a bit mask over its lattice; the compact index of an unknown is the
// count of unknowns before its word (an exclusive scan of the words' counts) plus those before
// it in the word.

// A coarser level's posts: the parents (col / 2, row / 2) of the finer level's unknowns.
__global__ void coarsen_kernel(const uint32_t* __restrict__ finePos, uint32_t n, uint32_t fineW,
                               uint32_t coarsePitch, uint32_t* __restrict__ coarseMask) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) {
        return;
    }
    const uint32_t p = finePos[k];
    const uint32_t col = (p % fineW) / 2, row = p / fineW / 2;
    atomicOr(&coarseMask[size_t(row) * coarsePitch + (col >> 5)], 1u << (col & 31u));
}

__global__ void word_counts_kernel(const uint32_t* __restrict__ mask, size_t words,
                                   uint32_t* __restrict__ counts) {
    const size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q < words) {
        counts[q] = __popc(mask[q]);
    }
}

// Each unknown's post, from its word's offset.
__global__ void positions_kernel(const uint32_t* __restrict__ mask,
                                 const uint32_t* __restrict__ offsets, size_t words,
                                 uint32_t pitch, uint32_t w, uint32_t* __restrict__ position) {
    const size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= words) {
        return;
    }
    uint32_t m = mask[q];
    uint32_t at = offsets[q];
    const uint32_t base = uint32_t(q / pitch) * w + uint32_t(q % pitch) * 32u;
    while (m != 0) {
        position[at++] = base + uint32_t(__ffs(int(m)) - 1);
        m &= m - 1u;
    }
}

// One level: its lattice, its unknowns and the operator's weights.
struct LevelView {
    uint32_t w, h, n, pitch;
    const uint32_t* mask;      // [pitch * h] 1 at the unknowns
    const uint32_t* offsets;   // [pitch * h] unknowns before each word
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

// The compact index of the post (c, r), or ~0u where it is not an unknown.
__device__ __forceinline__ uint32_t index_at(const LevelView& L, int c, int r) {
    const size_t q = size_t(r) * L.pitch + uint32_t(c >> 5);
    const uint32_t m = L.mask[q], b = uint32_t(c & 31);
    return (m >> b) & 1u ? L.offsets[q] + __popc(m & ((1u << b) - 1u)) : kNone;
}

__device__ __forceinline__ bool unknown_at(const LevelView& L, int c, int r) {
    return (L.mask[size_t(r) * L.pitch + uint32_t(c >> 5)] >> (c & 31)) & 1u;
}

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
                : index_at(L, c, r);
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
                : index_at(Cl, cs[j], rs[j]);
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
                    : index_at(F, fx, fy);
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
        return unknown_at(L, col + dc, row + dr)
                   ? 0.0
                   : double(field[size_t(row + dr) * L.w + uint32_t(col + dc)]);
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

// The start of a kernel launched by pdl_launch: wait for the kernels before it, then let the
// next one launch (a no-op for a plain launch).
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Damped Jacobi: xn = x + omega (b - A x) / diagonal; from x = 0 when `x` is null.
template <int kOrder, typename T>
__global__ void jacobi_kernel(const LevelView L, const T* __restrict__ b, const T* __restrict__ x,
                              T* __restrict__ xn, double omega, const CgState* cg) {
    pdl_begin();
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
    pdl_begin();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < L.n && !stopped(cg)) {
        r[k] = b[k] - apply_at<kOrder, T, T>(L, x, k);
    }
}

// Restriction, gathered: coarse unknown (C, R) takes 1/4 of each fine residual whose parent or
// parent's neighbor it is, weighted 3/4 or 1/4 per axis (the transfer weights 9/16, 3/16, 3/16,
// 1/16, seam_field.cpp:56).
template <typename Tf, typename Tc>
__global__ void restrict_kernel(const LevelView F, const LevelView Cl, const Tf* __restrict__ r,
                                Tc* __restrict__ b, const CgState* cg) {
    pdl_begin();
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
    pdl_begin();
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

// The block's sums of x and y into partial[block] and partial[kDotBlocks + block], as a fixed
// tree over 256 threads.
__device__ __forceinline__ void block_partials(double x, double y, double* __restrict__ partial) {
    __shared__ double s0[256], s1[256];
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

// Partial sums of a . b (and of c . d when given) per block (kDotBlocks blocks of 256 threads);
// summed by finish_kernel in a fixed order, so every run gives the same bits.
__global__ void dot_kernel(const double* __restrict__ a, const double* __restrict__ b,
                           const double* __restrict__ c, const double* __restrict__ d, uint32_t n,
                           double* __restrict__ partial, const CgState* cg) {
    pdl_begin();
    if (stopped(cg)) {
        return;
    }
    double x = 0.0, y = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        x += a[k] * b[k];
        if (c != nullptr) {
            y += c[k] * d[k];
        }
    }
    block_partials(x, y, partial);
}

// Ap = A p, with the partial sums of p . Ap.
template <int kOrder>
__global__ void apply_dot_kernel(const LevelView L, const double* __restrict__ p,
                                 double* __restrict__ ap, double* __restrict__ partial,
                                 const CgState* cg) {
    pdl_begin();
    if (stopped(cg)) {
        return;
    }
    double x = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < L.n;
         k += gridDim.x * blockDim.x) {
        const double a = apply_at<kOrder, double, double>(L, p, k);
        ap[k] = a;
        x += p[k] * a;
    }
    block_partials(x, 0.0, partial);
}

// The partial sums of r . r and r . z, z the V-cycle's result on the finest level (float).
__global__ void precondition_dots_kernel(const double* __restrict__ r,
                                         const float* __restrict__ z, uint32_t n,
                                         double* __restrict__ partial, const CgState* cg) {
    pdl_begin();
    if (stopped(cg)) {
        return;
    }
    double x = 0.0, y = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double rk = r[k];
        x += rk * rk;
        y += rk * double(z[k]);
    }
    block_partials(x, y, partial);
}

enum Then { kThenNothing = 0, kThenStep = 1, kThenNext = 2 };

// The block partials summed by one block of kDotBlocks threads as a fixed tree, so every run
// adds them in the same order; then, on the device state:
//   kThenStep, after p . Ap: the step, or the stop when the curvature is not positive or the
//     iterations are spent (PreconditionedCg, seam_field.cpp:519-527);
//   kThenNext, after r . r and r . z: the stop at the target residual, else the direction's
//     ratio (seam_field.cpp:532-542).
__global__ void finish_kernel(const double* __restrict__ partial, double* __restrict__ out,
                              CgState* cg, int then) {
    pdl_begin();
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
    if (threadIdx.x != 0) {
        return;
    }
    out[0] = s0[0];
    out[1] = s1[0];
    if (then == kThenStep) {
        const double curvature = s0[0];
        if (cg->iterations >= cg->maxIterations || !(cg->fit > 0.0) || !(curvature > 0.0)) {
            cg->done = 1u;
            return;
        }
        cg->step = cg->fit / curvature;
        cg->iterations += 1u;
    } else if (then == kThenNext) {
        if (sqrt(s0[0]) <= cg->target) {
            cg->done = 1u;
            return;
        }
        const double next = s1[0];
        cg->ratio = next / cg->fit;
        cg->fit = next;
    }
}

// x += step p, r -= step Ap; with `b0`, the finest level's right-hand side float(r) for the
// V-cycle, and with `x0` its first smoothing sweep from 0 (scale b).
__global__ void cg_update_kernel(double* __restrict__ x, double* __restrict__ r,
                                 const double* __restrict__ p, const double* __restrict__ ap,
                                 uint32_t n, float* __restrict__ b0, float* __restrict__ x0,
                                 float scale, const CgState* cg) {
    pdl_begin();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        const double step = cg->step;
        x[k] += step * p[k];
        const double rk = r[k] - step * ap[k];
        r[k] = rk;
        if (b0 != nullptr) {
            const float bk = float(rk);
            b0[k] = bk;
            if (x0 != nullptr) {
                x0[k] = scale * bk;
            }
        }
    }
}

// p = z + ratio p.
template <typename T>
__global__ void cg_direction_kernel(double* __restrict__ p, const T* __restrict__ z, uint32_t n,
                                    const CgState* cg) {
    pdl_begin();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        p[k] = double(z[k]) + cg->ratio * p[k];
    }
}

// The coarsest level's sweeps in one block, its iterates in shared memory: the same damped
// Jacobi steps as jacobi_kernel, a block barrier between sweeps.
constexpr uint32_t kCoarsestBlockPosts = 4096;

template <int kOrder>
__global__ void __launch_bounds__(1024) coarsest_kernel(const LevelView L,
                                                        const double* __restrict__ b,
                                                        double* __restrict__ x, double omega,
                                                        int sweeps, const CgState* cg) {
    pdl_begin();
    if (stopped(cg)) {
        return;
    }
    extern __shared__ double iterates[];
    double* cur = iterates;
    double* next = iterates + L.n;
    const double scale = omega / L.diagonal;
    for (int i = 0; i < sweeps; ++i) {
        for (uint32_t k = threadIdx.x; k < L.n; k += blockDim.x) {
            if (i == 0) {
                next[k] = scale * b[k];
            } else {
                const double r = b[k] - apply_at<kOrder, double, double>(L, cur, k);
                next[k] = cur[k] + scale * r;
            }
        }
        __syncthreads();
        double* t = cur;
        cur = next;
        next = t;
    }
    for (uint32_t k = threadIdx.x; k < L.n; k += blockDim.x) {
        x[k] = cur[k];
    }
}

template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ in, B* __restrict__ out, uint32_t n,
                               const CgState* cg) {
    pdl_begin();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !stopped(cg)) {
        out[k] = B(in[k]);
    }
}

template <typename T>
__global__ void copy_kernel(const T* __restrict__ in, T* __restrict__ out, uint32_t n,
                            const CgState* cg) {
    pdl_begin();
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
    Buffer mask, offsets, position, x, b, t;  // x, b, t: float (double on the coarsest level)
    Buffer nbr, parents, children;
};

// The seam calls' device scratch, one per device, grown as needed and kept across calls (no
// allocation, and so no device-wide synchronization of a free, on a call that fits).
struct Work {
    Buffer bits, count, scan, steps, rows, partial, dots;
    Buffer tileCounts, tileList, cg;
    Buffer cgX, cgR, cgP, cgAp, cgZ, rhs;
    Buffer hostIn, hostIn2, hostOut, hostOut2;  // device copies of host-memory arguments
    Level levels[kMaxLevels];
    ~Work() {
        for (Buffer* b : {&bits, &count, &scan, &steps, &rows, &partial, &dots, &tileCounts,
                          &tileList, &cg, &cgX, &cgR, &cgP, &cgAp, &cgZ, &rhs, &hostIn, &hostIn2,
                          &hostOut, &hostOut2}) {
            b->release();
        }
        for (Level& l : levels) {
            for (Buffer* b : {&l.mask, &l.offsets, &l.position, &l.x, &l.b, &l.t, &l.nbr,
                              &l.parents, &l.children}) {
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

// The level's compact index and positions from its unknown mask (`level.mask`, `pitch` words a
// row of a w x h lattice).
int compact(Work& wk, Level& level, uint32_t w, uint32_t h, uint32_t pitch, cudaStream_t s) {
    const size_t words = size_t(pitch) * h;
    uint32_t* offsets = nullptr;
    TG_CUDA(level.offsets.reserve((words + 1) * sizeof(uint32_t)), "allocation");
    offsets = static_cast<uint32_t*>(level.offsets.ptr);
    const uint32_t* mask = static_cast<const uint32_t*>(level.mask.ptr);
    word_counts_kernel<<<blocks_for(words), 256, 0, s>>>(mask, words, offsets);
    TG_CUDA(wk.scan.reserve(scan_scratch_words(uint32_t(words)) * sizeof(uint32_t)),
            "allocation");
    TG_CUDA(launch_exclusive_scan(offsets, uint32_t(words), static_cast<uint32_t*>(wk.scan.ptr),
                                  s),
            "scan");
    uint32_t total = 0;
    TG_CUDA(cudaMemcpyAsync(&total, offsets + words, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy to host");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    TG_CUDA(level.position.reserve(std::max<size_t>(total, 1) * sizeof(uint32_t)), "allocation");
    positions_kernel<<<blocks_for(words), 256, 0, s>>>(
        mask, offsets, words, pitch, w, static_cast<uint32_t*>(level.position.ptr));
    TG_CUDA(cudaGetLastError(), "compact launch");
    level.view.w = w;
    level.view.h = h;
    level.view.n = total;
    level.view.pitch = pitch;
    level.view.mask = mask;
    level.view.offsets = offsets;
    level.view.position = static_cast<const uint32_t*>(level.position.ptr);
    return TG_OK;
}

// Launches with programmatic dependent launch: the next kernel of the stream may start before
// this one ends; every kernel launched this way begins with pdl_begin(), which waits for the
// kernels before it (their writes visible) and lets the next one launch.
template <typename... K, typename... A>
cudaError_t pdl_launch(void (*kernel)(K...), dim3 grid, dim3 block, size_t shared,
                       cudaStream_t stream, A&&... args) {
    cudaLaunchConfig_t config{};
    config.gridDim = grid;
    config.blockDim = block;
    config.dynamicSmemBytes = shared;
    config.stream = stream;
    cudaLaunchAttribute attribute[1];
    attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[0].val.programmaticStreamSerializationAllowed = 1;
    config.attrs = attribute;
    config.numAttrs = 1;
    return cudaLaunchKernelEx(&config, kernel, std::forward<A>(args)...);
}

#define TG_PDL(...)                                          \
    do {                                                     \
        const cudaError_t e_ = pdl_launch(__VA_ARGS__);      \
        if (e_ != cudaSuccess) {                             \
            return ::tgb::api::cuda_fail(e_, "launch");      \
        }                                                    \
    } while (0)

#define TG_PDL_E(...)                                        \
    do {                                                     \
        const cudaError_t e_ = pdl_launch(__VA_ARGS__);      \
        if (e_ != cudaSuccess) {                             \
            return e_;                                       \
        }                                                    \
    } while (0)

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
        TG_PDL_E(jacobi_kernel<kOrder, double>, blocks_for(L.n), 256, 0, sv.s,
            L, static_cast<const double*>(b), static_cast<const double*>(x),
            static_cast<double*>(xn), sv.omega, sv.cg);
    } else {
        TG_PDL_E(jacobi_kernel<kOrder, float>, blocks_for(L.n), 256, 0, sv.s,
            L, static_cast<const float*>(b), static_cast<const float*>(x),
            static_cast<float*>(xn), sv.omega, sv.cg);
    }
    return cudaGetLastError();
}

cudaError_t copy_level(const Solver& sv, const void* from, void* to, uint32_t n, bool wide) {
    if (wide) {
        TG_PDL_E(copy_kernel<double>, blocks_for(n), 256, 0, sv.s,
            static_cast<const double*>(from),
                                                            static_cast<double*>(to), n, sv.cg);
    } else {
        TG_PDL_E(copy_kernel<float>, blocks_for(n), 256, 0, sv.s,
            static_cast<const float*>(from),
                                                           static_cast<float*>(to), n, sv.cg);
    }
    return cudaGetLastError();
}

// Where a level's first smoothing sweep of `sweeps` writes: the sweeps alternate between x and t
// and the last lands in x.
void* first_sweep_target(Level& L, int sweeps) {
    return sweeps % 2 == 1 ? L.x.ptr : L.t.ptr;
}

// The V-cycle from level `d` (VCycle, seam_field.cpp:423): an approximate solution of the level's
// operator for its b, from 0, into its x. `smoothed` sweeps of the first smoothing are done
// already (0 or 1, the first one landing where this one would put it). Sweeps alternate between
// x and t so that the last lands in x.
template <int kOrder>
int vcycle(Solver& sv, int d, int smoothed = 0) {
    Level& L = sv.wk->levels[d];
    const bool last = d + 1 == sv.levels;
    if (L.view.n == 0) {
        return TG_OK;
    }
    const int sweeps = last ? sv.coarsest : sv.sweeps;
    if (last && smoothed == 0 && L.view.n <= kCoarsestBlockPosts) {
        const uint32_t threads = std::min<uint32_t>(1024, (L.view.n + 31) / 32 * 32);
        TG_PDL(coarsest_kernel<kOrder>, 1, threads, size_t(L.view.n) * 16, sv.s,
            L.view, static_cast<const double*>(L.b.ptr), static_cast<double*>(L.x.ptr),
            sv.omega, sweeps, sv.cg);
        TG_CUDA(cudaGetLastError(), "coarsest launch");
        return TG_OK;
    }
    void* cur = smoothed > 0 ? first_sweep_target(L, sweeps) : nullptr;
    for (int i = smoothed; i < sweeps; ++i) {
        void* next = (sweeps - i) % 2 == 1 ? L.x.ptr : L.t.ptr;
        TG_CUDA(jacobi<kOrder>(sv, L.view, L.b.ptr, cur, next, last), "jacobi");
        cur = next;
    }
    if (last) {
        return TG_OK;
    }
    Level& C = sv.wk->levels[d + 1];
    const bool coarseLast = d + 2 == sv.levels;
    // residual into t, restricted into the coarse b
    TG_PDL(residual_kernel<kOrder, float>, blocks_for(L.view.n), 256, 0, sv.s,
        L.view, static_cast<const float*>(L.b.ptr), static_cast<const float*>(L.x.ptr),
        static_cast<float*>(L.t.ptr), sv.cg);
    if (coarseLast) {
        TG_PDL(restrict_kernel<float, double>, blocks_for(C.view.n), 256, 0, sv.s,
            L.view, C.view, static_cast<const float*>(L.t.ptr), static_cast<double*>(C.b.ptr),
            sv.cg);
    } else {
        TG_PDL(restrict_kernel<float, float>, blocks_for(C.view.n), 256, 0, sv.s,
            L.view, C.view, static_cast<const float*>(L.t.ptr), static_cast<float*>(C.b.ptr),
            sv.cg);
    }
    TG_CUDA(cudaGetLastError(), "restrict launch");
    if (int st = vcycle<kOrder>(sv, d + 1)) {
        return st;
    }
    if (coarseLast) {
        TG_PDL(prolong_kernel<double, float>, blocks_for(L.view.n), 256, 0, sv.s,
            L.view, C.view, static_cast<const double*>(C.x.ptr), static_cast<float*>(L.x.ptr),
            sv.cg);
    } else {
        TG_PDL(prolong_kernel<float, float>, blocks_for(L.view.n), 256, 0, sv.s,
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
    TG_PDL(convert_kernel<double, float>, blocks_for(n), 256, 0, sv.s,
        r, static_cast<float*>(L0.b.ptr), n, sv.cg);
    if (int st = vcycle<kOrder>(sv, 0)) {
        return st;
    }
    TG_PDL(convert_kernel<float, double>, blocks_for(n), 256, 0, sv.s,
        static_cast<const float*>(L0.x.ptr), z, n, sv.cg);
    TG_CUDA(cudaGetLastError(), "convert launch");
    return TG_OK;
}

// a . b and c . d (c may be null) into `out` on the device, then `then` on the state.
cudaError_t dots(const Solver& sv, const double* a, const double* b, const double* c,
                 const double* d, uint32_t n, double* out, CgState* cg = nullptr,
                 int then = kThenNothing) {
    TG_PDL_E(dot_kernel, kDotBlocks, 256, 0, sv.s,
        a, b, c, d, n,
                                             static_cast<double*>(sv.wk->partial.ptr), sv.cg);
    TG_PDL_E(finish_kernel, 1, kDotBlocks, 0, sv.s,
        static_cast<const double*>(sv.wk->partial.ptr),
                                              out, cg, then);
    return cudaGetLastError();
}

// Iterations launched between looks at whether the conjugate gradients stopped.
constexpr int kIterationsPerGraph = 4;

// One iteration of PreconditionedCg (seam_field.cpp:517-542), every scalar on the device. With
// more than one level, the update writes the finest level's right-hand side and first sweep, and
// z stays the finest level's float iterate: the dots and the direction read it there.
template <int kOrder>
int iteration(Solver& sv, CgState* cg) {
    Work& wk = *sv.wk;
    Level& L0 = wk.levels[0];
    const uint32_t n = L0.view.n;
    double* x = static_cast<double*>(wk.cgX.ptr);
    double* r = static_cast<double*>(wk.cgR.ptr);
    double* p = static_cast<double*>(wk.cgP.ptr);
    double* ap = static_cast<double*>(wk.cgAp.ptr);
    double* z = static_cast<double*>(wk.cgZ.ptr);
    double* partial = static_cast<double*>(wk.partial.ptr);
    TG_PDL(apply_dot_kernel<kOrder>, kDotBlocks, 256, 0, sv.s,
        L0.view, p, ap, partial, cg);
    TG_PDL(finish_kernel, 1, kDotBlocks, 0, sv.s,
        partial, cg_dots(cg), cg, kThenStep);
    if (sv.levels == 1) {
        TG_PDL(cg_update_kernel, blocks_for(n), 256, 0, sv.s,
            x, r, p, ap, n, nullptr, nullptr, 0.0f,
                                                          cg);
        if (int st = precondition<kOrder>(sv, r, z)) {
            return st;
        }
        TG_CUDA(dots(sv, r, r, r, z, n, cg_dots(cg), cg, kThenNext), "dot launch");
        TG_PDL(cg_direction_kernel<double>, blocks_for(n), 256, 0, sv.s,
            p, z, n, cg);
        TG_CUDA(cudaGetLastError(), "iteration launch");
        return TG_OK;
    }
    const float scale = float(sv.omega / L0.view.diagonal);
    TG_PDL(cg_update_kernel, blocks_for(n), 256, 0, sv.s,
        x, r, p, ap, n, static_cast<float*>(L0.b.ptr),
        static_cast<float*>(first_sweep_target(L0, sv.sweeps)), scale, cg);
    if (int st = vcycle<kOrder>(sv, 0, 1)) {
        return st;
    }
    const float* z0 = static_cast<const float*>(L0.x.ptr);
    TG_PDL(precondition_dots_kernel, kDotBlocks, 256, 0, sv.s,
        r, z0, n, partial, cg);
    TG_PDL(finish_kernel, 1, kDotBlocks, 0, sv.s,
        partial, cg_dots(cg), cg, kThenNext);
    TG_PDL(cg_direction_kernel<float>, blocks_for(n), 256, 0, sv.s,
        p, z0, n, cg);
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
    Events ev;
    if (ev.create() != cudaSuccess) {
        return finish(fail(TG_ERROR_CUDA, "event"));
    }
    TG_CUDA(cudaEventRecord(ev.e[0], s), "event");
    // The field is 0 without a seam, and when the earlier source has data at every post or at
    // none.
    auto empty = [&]() {
        TG_CUDA(cudaMemsetAsync(dField, 0, n * 4, s), "memset");
        return finish(TG_OK);
    };
    if (o.mode == 0u) {
        return empty();
    }
    int sms = 0;
    TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->ordinal),
            "attribute");
    const uint32_t pitch = (width + 31) / 32;
    const size_t words = size_t(pitch) * height;
    TG_CUDA(wk.bits.reserve(words * 4), "allocation");
    TG_CUDA(wk.count.reserve(8), "allocation");
    TG_CUDA(cudaMemsetAsync(wk.count.ptr, 0, 8, s), "memset");
    uint32_t* bits = static_cast<uint32_t*>(wk.bits.ptr);
    pack_data_kernel<<<uint32_t(std::min<size_t>(
                           blocks_for((words + kPackWords - 1) / kPackWords * 32), size_t(sms) * 8)),
                       256, 0, s>>>(dData, width, height, pitch, bits,
                                    static_cast<unsigned long long*>(wk.count.ptr));
    unsigned long long withData = 0;
    TG_CUDA(cudaMemcpyAsync(&withData, wk.count.ptr, 8, cudaMemcpyDeviceToHost, s), "copy");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    if (withData == 0 || withData == n) {
        return empty();
    }
    // Distances to the nearest post with data matter up to the reach (Height, Slope) or the
    // width (Feather).
    const bool feather = o.mode == 1u;
    const double reach = feather ? o.width : 3.0 * o.decay_length;  // kSeamReachDecays
    const float cap =
        float(reach) < reach ? std::nextafter(float(reach), INFINITY) : float(reach);
    // Halo of the tiled passes: a distance at most `cap` reaches cap / dx columns, cap / dy rows.
    const int mx = int(std::min(std::ceil(double(cap) / dx) + 2.0, double(width)));
    const int my = int(std::min(std::ceil(double(cap) / dy) + 2.0, double(height)));
    const int halo = std::max(mx, my);
    const int ts = halo <= 128 ? 64 : std::min(1024, (halo / 2 + 31) / 32 * 32);
    const uint32_t tilesX = (width + ts - 1) / ts, tilesY = (height + ts - 1) / ts;
    const size_t tiles = size_t(tilesX) * tilesY;
    TG_CUDA(wk.tileCounts.reserve(tiles * 4), "allocation");
    TG_CUDA(wk.tileList.reserve(tiles * 4 + 4), "allocation");
    uint32_t* counts = static_cast<uint32_t*>(wk.tileCounts.ptr);
    uint32_t* list = static_cast<uint32_t*>(wk.tileList.ptr);
    TG_CUDA(cudaMemsetAsync(counts, 0, tiles * 4, s), "memset");
    TG_CUDA(cudaMemsetAsync(list, 0, 4, s), "memset");
    // The band's differences (every post of the field written), and the posts with data per
    // tile.
    BandBits bb{bits, dDiff, dField, counts, width, height, pitch, ts, tilesX};
    const size_t bandWarps = size_t((pitch + 31) / 32) * ((height + kBandRows - 1) / kBandRows);
    band_bits_kernel<<<blocks_for(bandWarps * 32), 256, 0, s>>>(bb);
    TG_CUDA(cudaGetLastError(), "band launch");
    active_tiles_kernel<<<blocks_for(tiles), 256, 0, s>>>(
        counts, width, height, ts, tilesX, tilesY, (mx + ts - 1) / ts, (my + ts - 1) / ts,
        list + 1, list);
    uint32_t active = 0;
    TG_CUDA(cudaMemcpyAsync(&active, list, 4, cudaMemcpyDeviceToHost, s), "copy");
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    Level& L0 = wk.levels[0];
    if (!feather) {
        TG_CUDA(L0.mask.reserve(words * 4), "allocation");
        TG_CUDA(cudaMemsetAsync(L0.mask.ptr, 0, words * 4, s), "memset");
    }
    if (active > 0) {
        DistanceWarps p{};
        p.bits = bits;
        p.field = feather ? dField : nullptr;
        p.w = width;
        p.h = height;
        p.pitch = pitch;
        p.dx = float(dx);
        p.dy = float(dy);
        p.diagonal = float(std::hypot(dx, dy));
        p.ts = ts;
        p.mx = mx;
        p.my = my;
        p.tilesX = tilesX;
        p.list = list + 1;
        p.count = list;
        p.unknown = feather ? nullptr : static_cast<uint32_t*>(L0.mask.ptr);
        p.reach = reach;
        p.feather = feather ? dField : nullptr;
        p.width = o.width;
        // A window is at most ts + 2 mx columns and ts + 2 my rows; the backward pass covers
        // its rows from the tile's first.
        const int carriedCopies = feather ? 2 : 1;
        p.rowFloats = int(std::min<size_t>(size_t(ts) + 2 * size_t(mx), width));
        const size_t bandsBelow = (std::min<size_t>(size_t(ts) + my, height) + 31) / 32;
        p.scratchFloats = size_t(carriedCopies) * bandsBelow * (size_t(p.rowFloats) + 62) * 32;
        const size_t rowBytes = size_t(p.rowFloats) * 4 * carriedCopies;
        const bool sharedRows = rowBytes * kDistanceWarps <= kRowSharedBytes;
        const size_t shared = sharedRows ? rowBytes * kDistanceWarps : 0;
        auto kernel = feather ? (sharedRows ? distance_warp_kernel<true, true>
                                            : distance_warp_kernel<true, false>)
                              : (sharedRows ? distance_warp_kernel<false, true>
                                            : distance_warp_kernel<false, false>);
        TG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(shared)),
                "shared memory attribute");
        int perSm = 0;
        TG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel,
                                                              32 * kDistanceWarps, shared),
                "occupancy");
        size_t slots = size_t(std::max(1, perSm)) * size_t(sms) * kDistanceWarps;
        slots = std::min<size_t>(slots, active);
        slots = std::min<size_t>(
            slots, std::max<size_t>(1, kScratchBytes / (p.scratchFloats * 4 + rowBytes)));
        p.slots = uint32_t(slots);
        TG_CUDA(wk.steps.reserve(slots * p.scratchFloats * 4), "allocation");
        p.scratch = static_cast<float*>(wk.steps.ptr);
        if (!sharedRows) {
            TG_CUDA(wk.rows.reserve(slots * rowBytes), "allocation");
            p.rows = static_cast<float*>(wk.rows.ptr);
        }
        kernel<<<uint32_t((slots + kDistanceWarps - 1) / kDistanceWarps), 32 * kDistanceWarps,
                 shared, s>>>(p);
        TG_CUDA(cudaGetLastError(), "distance launch");
    }
    if (feather) {
        return finish(TG_OK);
    }
    // The unknowns of each level.
    const int order = o.mode == 3u ? 2 : 1;
    const double screening = 1.0 / (o.decay_length * o.decay_length);
    int levels = 0;
    uint32_t lw = width, lh = height, lp = pitch;
    double ldx = dx, ldy = dy;
    for (; levels < int(o.levels); ++levels) {
        Level& L = wk.levels[levels];
        if (levels > 0) {
            const Level& F = wk.levels[levels - 1];
            lw = (lw + 1) / 2;
            lh = (lh + 1) / 2;
            lp = (lw + 31) / 32;
            ldx *= 2.0;
            ldy *= 2.0;
            TG_CUDA(L.mask.reserve(size_t(lp) * lh * 4), "allocation");
            TG_CUDA(cudaMemsetAsync(L.mask.ptr, 0, size_t(lp) * lh * 4, s), "memset");
            coarsen_kernel<<<blocks_for(F.view.n), 256, 0, s>>>(
                F.view.position, F.view.n, F.view.w, lp, static_cast<uint32_t*>(L.mask.ptr));
            TG_CUDA(cudaGetLastError(), "coarsen launch");
        }
        if (int st = compact(wk, L, lw, lh, lp, s)) {
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
    for (auto kernel : {coarsest_kernel<1>, coarsest_kernel<2>}) {
        TG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(kCoarsestBlockPosts * 16)),
                "shared memory attribute");
    }
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
