// fBm noise sources and noise layers over a grid (SyntheticSource::FillSamples,
// src/sources/synthetic_source.cpp:87; NoiseLayer::ApplySamples, src/layers/noise_layer.cpp:95).
//
// Compiled with -fmad=false: positions (double) and the lattice math (float) round exactly as the
// reference's -ffp-contract=off build does, so heights carry the reference CPU path's bits.
//
// The kernel is ALU-bound (about 1.6k integer and float operations per cell for 8 Perlin
// octaves, 4 bytes written). Each thread evaluates kRowsPerThread cells of one column, so a warp
// covers 32 consecutive columns and every store is a full 128-byte line.
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

// One enabled Perlin fBm fractal without a warp: the configurations' source, the hot case.
struct SingleFbm {
    uint32_t seed;
    float wavelength, amplitude, lacunarity, gain;
    int octaves;
};

template <bool kSingle>
__global__ void __launch_bounds__(kBlockX* kBlockY)
    noise_kernel(const FractalStack stack, const SingleFbm fbm, const Grid grid,
                 const Positions at, const bool fill, const float elevation, const NoData nodata,
                 float* __restrict__ heights) {
    const uint32_t col = blockIdx.x * kBlockX + threadIdx.x;
    const uint32_t row0 = (blockIdx.y * kBlockY + threadIdx.y) * kRowsPerThread;
    if (col >= grid.width) {
        return;
    }
#pragma unroll
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
        float n;
        if (kSingle) {
            // EvaluateFractals of one enabled fractal: amplitude * (unit-amplitude fBm).
            n = fbm.amplitude * noise::perlin_fbm2(x, y, fbm.seed, fbm.wavelength, 1.0f,
                                                   fbm.octaves, fbm.lacunarity, fbm.gain);
        } else {
            n = noise::evaluate_stack(x, y, stack.fractals, stack.count);
        }
        heights[i] = base + n;
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

cudaError_t launch_noise(const FractalStack& stack, const Grid& grid, const Positions& at,
                         bool fill, float elevation, NoData nodata, float* heights,
                         cudaStream_t stream) {
    if (grid.width == 0 || grid.height == 0) {
        return cudaSuccess;
    }
    // The fast path: exactly one enabled fractal, Perlin fBm, no warp.
    SingleFbm fbm{};
    int enabled = 0;
    const Fractal* only = nullptr;
    for (uint32_t i = 0; i < stack.count && i < kMaxFractals; ++i) {
        if (stack.fractals[i].enabled) {
            ++enabled;
            only = &stack.fractals[i];
        }
    }
    const bool single = enabled == 1 && only->basis == kBasisPerlin && only->type == kTypeFbm &&
                        !(only->warpAmplitude > 0.0f);
    if (single) {
        fbm = SingleFbm{only->seed, only->wavelength, only->amplitude, only->lacunarity,
                        only->gain, only->octaves};
    }
    const dim3 block(kBlockX, kBlockY);
    const uint32_t rowsPerBlock = kBlockY * kRowsPerThread;
    const dim3 blocks((grid.width + kBlockX - 1) / kBlockX,
                      (grid.height + rowsPerBlock - 1) / rowsPerBlock);
    if (single) {
        noise_kernel<true><<<blocks, block, 0, stream>>>(stack, fbm, grid, at, fill, elevation,
                                                         nodata, heights);
    } else {
        noise_kernel<false><<<blocks, block, 0, stream>>>(stack, fbm, grid, at, fill, elevation,
                                                          nodata, heights);
    }
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
