// fBm noise sources and noise layers over a grid (SyntheticSource::FillSamples,
// src/sources/synthetic_source.cpp:87; NoiseLayer::ApplySamples, src/layers/noise_layer.cpp:95).
//
// Compiled with -fmad=false: positions (double) and the lattice math (float) round exactly as the
// reference's -ffp-contract=off build does, so heights carry the reference CPU path's bits.
//
// The kernels are ALU-bound (about 1.5k integer and float operations per cell for 8 Perlin
// octaves, 4 bytes written). Each thread evaluates several cells of one column, so a warp covers
// 32 consecutive columns and every store is a full 128-byte line.
#include "kernels.h"
#include "noise_math.cuh"

namespace tgb {
namespace {

constexpr int kRowsPerThread = 4;
constexpr int kBlockX = 32;
constexpr int kBlockY = 8;

__device__ __forceinline__ bool is_nodata(NoData nd, float h) {
    if (nd.mode == 1u) {
        return isnan(h);
    }
    return nd.mode != 0u && h == nd.value;
}

// The float x of a column's cell centers measured from the origin (src/gpu/kernel.cpp:56-62):
// computed in double as Raster::CellCenter does, then narrowed.
__device__ __forceinline__ float column_x(const Grid& g, const Positions& at, uint32_t col,
                                          uint32_t row) {
    if (at.xs != nullptr) {
        return at.xs[col];
    }
    const double x = g.originX + (double(col) + 0.5) * g.pixelWidth +
                     (double(row) + 0.5) * g.rowRotation;
    return float(x - at.originX);
}

__device__ __forceinline__ float row_y(const Grid& g, const Positions& at, uint32_t col,
                                       uint32_t row) {
    if (at.ys != nullptr) {
        return at.ys[row];
    }
    const double y = g.originY + (double(col) + 0.5) * g.colRotation +
                     (double(row) + 0.5) * g.pixelHeight;
    return float(y - at.originY);
}

// One enabled Perlin fBm fractal without a warp, the configurations' source: its per-octave
// constants are computed once on the host, with the same float recurrences Fractal2 runs per
// cell (fractal.h:219-240), so each cell performs exactly the reference's operations on them.
constexpr int kMaxOctaves = 32;
struct Octaves {
    int count;
    float amplitude;
    float total;                       // sum of the weights
    uint32_t seedTerm[kMaxOctaves];    // octave seed, through pcg3d's first LCG step
    float ox[kMaxOctaves], oy[kMaxOctaves];
    float frequency[kMaxOctaves], weight[kMaxOctaves];
    float tc[kMaxOctaves], ts[kMaxOctaves];
};

constexpr uint32_t kLcgA = 1664525u, kLcgC = 1013904223u;

// pcg3d's x word for a corner whose first-step terms are already applied (hash.h:40-57).
__device__ __forceinline__ uint32_t corner_from_terms(uint32_t x, uint32_t y, uint32_t z) {
    x += y * z;
    y += z * x;
    z += x * y;
    x ^= x >> 16u;
    y ^= y >> 16u;
    z ^= z >> 16u;
    return x + y * z;
}

constexpr int kFbmRows = 8;  // rows per thread in the fBm kernel

// The fBm source: octave-outer over kFbmRows cells of a column, reusing a lattice cell's four
// corner hashes from the row above when the cell is the same (most rows, at broad octaves).
__global__ void __launch_bounds__(kBlockX* kBlockY)
    fbm_kernel(const Octaves oct, const Grid grid, const Positions at, const bool fill,
               const float elevation, const NoData nodata, float* __restrict__ heights) {
    const uint32_t col = blockIdx.x * kBlockX + threadIdx.x;
    const uint32_t row0 = (blockIdx.y * kBlockY + threadIdx.y) * kFbmRows;
    if (col >= grid.width || row0 >= grid.height) {
        return;
    }
    const int rows = min(kFbmRows, int(grid.height - row0));
    float xs[kFbmRows], ys[kFbmRows], sum[kFbmRows];
#pragma unroll
    for (int r = 0; r < kFbmRows; ++r) {
        const uint32_t row = row0 + min(r, rows - 1);
        xs[r] = column_x(grid, at, col, row);
        ys[r] = row_y(grid, at, col, row);
        sum[r] = 0.0f;
    }
    for (int o = 0; o < oct.count; ++o) {
        const float tc = oct.tc[o], ts = oct.ts[o], f = oct.frequency[o];
        const float ox = oct.ox[o], oy = oct.oy[o], w = oct.weight[o];
        const uint32_t sz = oct.seedTerm[o];
        int32_t cx = INT32_MIN, cy = INT32_MIN;
        uint32_t h00 = 0, h10 = 0, h01 = 0, h11 = 0;
#pragma unroll
        for (int r = 0; r < kFbmRows; ++r) {
            // Fractal2's rotation and lattice position, then PerlinNoise2 (perlin.h:72-98).
            const float rx = xs[r] * tc - ys[r] * ts;
            const float ry = xs[r] * ts + ys[r] * tc;
            const noise::Cell2 c = noise::split2(rx * f + ox, ry * f + oy);
            if (c.ix != cx || c.iy != cy) {
                cx = c.ix;
                cy = c.iy;
                const uint32_t ax0 = uint32_t(c.ix) * kLcgA + kLcgC, ax1 = ax0 + kLcgA;
                const uint32_t ay0 = uint32_t(c.iy) * kLcgA + kLcgC, ay1 = ay0 + kLcgA;
                h00 = corner_from_terms(ax0, ay0, sz);
                h10 = corner_from_terms(ax1, ay0, sz);
                h01 = corner_from_terms(ax0, ay1, sz);
                h11 = corner_from_terms(ax1, ay1, sz);
            }
            const float n00 = noise::gradient2(h00, c.fx, c.fy);
            const float n10 = noise::gradient2(h10, c.fx - 1.0f, c.fy);
            const float n01 = noise::gradient2(h01, c.fx, c.fy - 1.0f);
            const float n11 = noise::gradient2(h11, c.fx - 1.0f, c.fy - 1.0f);
            const float u = noise::fade(c.fx);
            const float v = noise::fade(c.fy);
            const float n = 1.41421356237309505f *
                            noise::lerp(v, noise::lerp(u, n00, n10), noise::lerp(u, n01, n11));
            sum[r] += w * n;
        }
    }
#pragma unroll
    for (int r = 0; r < kFbmRows; ++r) {
        if (r >= rows) {
            break;
        }
        const size_t i = size_t(row0 + r) * grid.width + col;
        float base = elevation;
        if (!fill) {
            base = heights[i];
            if (is_nodata(nodata, base)) {
                continue;
            }
        }
        // EvaluateFractals of one enabled fractal: amplitude * (1 * sum / total).
        heights[i] = base + oct.amplitude * (1.0f * sum[r] / oct.total);
    }
}

// Any stack of fractals (bases, types, blends, warps), cell by cell.
__global__ void __launch_bounds__(kBlockX* kBlockY)
    noise_kernel(const FractalStack stack, const Grid grid, const Positions at, const bool fill,
                 const float elevation, const NoData nodata, float* __restrict__ heights) {
    const uint32_t col = blockIdx.x * kBlockX + threadIdx.x;
    const uint32_t row0 = (blockIdx.y * kBlockY + threadIdx.y) * kRowsPerThread;
    if (col >= grid.width) {
        return;
    }
    for (int r = 0; r < kRowsPerThread; ++r) {
        const uint32_t row = row0 + r;
        if (row >= grid.height) {
            return;
        }
        const size_t i = size_t(row) * grid.width + col;
        float base = elevation;
        if (!fill) {
            base = heights[i];
            if (is_nodata(nodata, base)) {
                continue;
            }
        }
        const float x = column_x(grid, at, col, row);
        const float y = row_y(grid, at, col, row);
        heights[i] = base + noise::evaluate_stack(x, y, stack.fractals, stack.count);
    }
}

// Per point: PcgHash(i), Pcg3dHash((x bits, y bits, seed)), then Perlin, simplex, value, Worley
// F1/F2/value, and Perlin fBm / ridged / billow / hybrid (seed `seed`) at (x, y).
__global__ void noise_probe_kernel(const float* __restrict__ xy, uint32_t n, uint32_t seed,
                                   uint32_t* __restrict__ hashes, float* __restrict__ values) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const float x = xy[2 * i], y = xy[2 * i + 1];
    hashes[4 * i] = noise::pcg(i);
    const noise::U3 h = noise::pcg3d(noise::U3{__float_as_uint(x), __float_as_uint(y), seed});
    hashes[4 * i + 1] = h.x;
    hashes[4 * i + 2] = h.y;
    hashes[4 * i + 3] = h.z;
    float* v = values + 12 * i;
    v[0] = noise::perlin2(x, y, seed);
    v[1] = noise::simplex2(x, y, seed);
    v[2] = noise::value2(x, y, seed);
    const noise::WorleyD w = noise::worley2(x, y, seed);
    v[3] = w.f1;
    v[4] = w.f2;
    v[5] = w.value;
    FractalParams p{seed, 1000.0f, 100.0f, 8, 2.0f, 0.5f, kBasisPerlin, kTypeFbm, 1.0f};
    v[6] = noise::fractal2(x, y, p);
    p.type = kTypeRidged;
    v[7] = noise::fractal2(x, y, p);
    p.type = kTypeBillow;
    v[8] = noise::fractal2(x, y, p);
    p.type = kTypeHybrid;
    v[9] = noise::fractal2(x, y, p);
    v[10] = noise::perlin3(x, y, 0.5f * (x - y), seed);
    v[11] = noise::perlin_fbm3_float(x, y, 0.25f * x, seed, 3, 0.5f);
}

}  // namespace

// A SyntheticSource on a sphere (SyntheticSource::NoiseAt with FractalStackAt on a body,
// surface_noise.cpp:14-17): each cell center's position R (cos lat cos lon, cos lat sin lon,
// sin lat) (UnitVector, surface.cpp:45), from the host's cosines and sines of each column's
// longitude and each row's latitude, then the stack in 3D.
__global__ void noise_body_kernel(const FractalStack stack, float elevation, uint32_t width,
                                  uint32_t height, const double* __restrict__ lons,
                                  const double* __restrict__ lats, double radius,
                                  float* __restrict__ heights) {
    const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= width || row >= height) {
        return;
    }
    const double cosLon = lons[2 * col], sinLon = lons[2 * col + 1];
    const double cosLat = lats[2 * row], sinLat = lats[2 * row + 1];
    const double x = cosLat * cosLon * radius;
    const double y = cosLat * sinLon * radius;
    const double z = sinLat * radius;
    heights[size_t(row) * width + col] =
        elevation + noise::evaluate_stack3(x, y, z, stack.fractals, stack.count);
}

cudaError_t launch_noise_body(const FractalStack& stack, float elevation, uint32_t width,
                              uint32_t height, const double* lons, const double* lats,
                              double radius, float* heights, cudaStream_t stream) {
    if (width == 0 || height == 0) {
        return cudaSuccess;
    }
    const dim3 block(32, 4);
    const dim3 grid((width + 31) / 32, (height + 3) / 4);
    noise_body_kernel<<<grid, block, 0, stream>>>(stack, elevation, width, height, lons, lats,
                                                  radius, heights);
    return cudaGetLastError();
}

cudaError_t launch_noise(const FractalStack& stack, const Grid& grid, const Positions& at,
                         bool fill, float elevation, NoData nodata, float* heights,
                         cudaStream_t stream) {
    if (grid.width == 0 || grid.height == 0) {
        return cudaSuccess;
    }
    // The fast path: exactly one enabled fractal, Perlin fBm, no warp.
    int enabled = 0;
    const Fractal* only = nullptr;
    for (uint32_t i = 0; i < stack.count && i < kMaxFractals; ++i) {
        if (stack.fractals[i].enabled) {
            ++enabled;
            only = &stack.fractals[i];
        }
    }
    const bool single = enabled == 1 && only->basis == kBasisPerlin && only->type == kTypeFbm &&
                        !(only->warpAmplitude > 0.0f) && only->octaves <= kMaxOctaves;
    const dim3 block(kBlockX, kBlockY);
    if (single) {
        // Fractal2's per-octave values, in its order of float operations (fractal.h:219-240);
        // this unit is built without contraction, so they round as on the reference's CPU.
        Octaves oct{};
        oct.count = only->octaves;
        oct.amplitude = only->amplitude;
        float frequency = 1.0f / only->wavelength;
        float tc = 1.0f, ts = 0.0f, weight = 1.0f, total = 0.0f;
        for (int o = 0; o < only->octaves; ++o) {
            uint32_t v[3] = {only->seed, uint32_t(o), 0u};
            v[0] = v[0] * kLcgA + kLcgC;
            v[1] = v[1] * kLcgA + kLcgC;
            v[2] = v[2] * kLcgA + kLcgC;
            v[0] += v[1] * v[2];
            v[1] += v[2] * v[0];
            v[2] += v[0] * v[1];
            v[0] ^= v[0] >> 16u;
            v[1] ^= v[1] >> 16u;
            v[2] ^= v[2] >> 16u;
            v[0] += v[1] * v[2];
            v[1] += v[2] * v[0];
            v[2] += v[0] * v[1];
            oct.seedTerm[o] = v[0] * kLcgA + kLcgC;  // the octave seed's first LCG step
            oct.ox[o] = float(v[1] >> 8u) * 0x1p-24f;
            oct.oy[o] = float(v[2] >> 8u) * 0x1p-24f;
            oct.frequency[o] = frequency;
            oct.tc[o] = tc;
            oct.ts[o] = ts;
            oct.weight[o] = weight;
            total += weight;
            weight *= only->gain;
            frequency *= only->lacunarity;
            const float nc = tc * TGB_TURN_COS - ts * TGB_TURN_SIN;
            ts = ts * TGB_TURN_COS + tc * TGB_TURN_SIN;
            tc = nc;
        }
        oct.total = total;
        const uint32_t rowsPerBlock = kBlockY * kFbmRows;
        const dim3 blocks((grid.width + kBlockX - 1) / kBlockX,
                          (grid.height + rowsPerBlock - 1) / rowsPerBlock);
        fbm_kernel<<<blocks, block, 0, stream>>>(oct, grid, at, fill, elevation, nodata, heights);
        return cudaGetLastError();
    }
    const uint32_t rowsPerBlock = kBlockY * kRowsPerThread;
    const dim3 blocks((grid.width + kBlockX - 1) / kBlockX,
                      (grid.height + rowsPerBlock - 1) / rowsPerBlock);
    noise_kernel<<<blocks, block, 0, stream>>>(stack, grid, at, fill, elevation, nodata, heights);
    return cudaGetLastError();
}

cudaError_t launch_noise_probe(const float* xy, uint32_t n, uint32_t seed, uint32_t* hashes,
                               float* values, cudaStream_t stream) {
    if (n == 0) {
        return cudaSuccess;
    }
    noise_probe_kernel<<<(n + 127) / 128, 128, 0, stream>>>(xy, n, seed, hashes, values);
    return cudaGetLastError();
}

}  // namespace tgb
