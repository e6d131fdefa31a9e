// Device-side lattice noise: PCG hashes, Perlin / simplex / value / Worley bases, fractal octave
// loops and fractal stacks, as TerrainGen's noise headers define them
// (include/terraingen/noise/{hash,lattice,perlin,simplex,value,worley,fractal,fractals}.h).
//
// Bit-exactness contract: the hashes, key layouts and lattice splits are integer or exactly
// rounded float work. A translation unit compiled with floating-point contraction off
// (-fmad=false, as noise.cu is), matching the reference's -ffp-contract=off
// (CMakeLists.txt:36-37), gets the reference CPU path's bits: only +, -, *, /, floor and sqrt
// appear, all IEEE-rounded on the GPU. Units that allow contraction (crater shaping) get values
// within a few ulp.
#pragma once

#include <stdint.h>

#include "layouts.h"

namespace tgb {
namespace noise {

// std::min / std::max / std::clamp with their exact comparison order, so NaNs and signed zeros
// resolve as they do on the CPU.
__device__ __forceinline__ float smin(float a, float b) {
    return b < a ? b : a;
}
__device__ __forceinline__ float smax(float a, float b) {
    return a < b ? b : a;
}
__device__ __forceinline__ float sclamp(float v, float lo, float hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

struct U3 {
    uint32_t x, y, z;
};

// PCG-RXS-M-XS over one LCG step (hash.h:33).
__device__ __forceinline__ uint32_t pcg(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

// The pcg3d mix of three words (hash.h:40).
__device__ __forceinline__ U3 pcg3d(U3 v) {
    v.x = v.x * 1664525u + 1013904223u;
    v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u;
    v.x += v.y * v.z;
    v.y += v.z * v.x;
    v.z += v.x * v.y;
    v.x ^= v.x >> 16u;
    v.y ^= v.y >> 16u;
    v.z ^= v.z >> 16u;
    v.x += v.y * v.z;
    v.y += v.z * v.x;
    v.z += v.x * v.y;
    return v;
}

// Top 24 bits of a hash as a float in [0, 1) (hash.h:60).
__device__ __forceinline__ float unit(uint32_t h) {
    return float(h >> 8u) * 0x1p-24f;
}

__device__ __forceinline__ float fade(float t) {  // lattice.h:79
    return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f);
}

__device__ __forceinline__ float lerp(float t, float a, float b) {  // lattice.h:84
    return a + t * (b - a);
}

// Dot product with one of eight 2D gradients picked by the corner hash's low bits
// (perlin.h:17).
__device__ __forceinline__ float gradient2(uint32_t hash, float x, float y) {
    const float kInvSqrt2 = 0.707106781186547524f;
    const uint32_t h = hash & 7u;
    const float axis = (h & 2u) != 0u ? y : x;
    const float sx = h == 5u ? -x : x;
    const float sy = h == 6u ? -y : y;
    const float sum = sx + sy;
    const float diagonal = (h == 7u ? -sum : sum) * kInvSqrt2;
    return h < 4u ? ((h & 1u) != 0u ? -axis : axis) : diagonal;
}

// Hash of a 2D lattice corner keyed (x, y, seed) (perlin.h:31, lattice.h:94).
__device__ __forceinline__ uint32_t corner2(uint32_t ix, uint32_t iy, uint32_t seed) {
    return pcg3d(U3{ix, iy, seed}).x;
}

// 2D improved Perlin noise of a lattice cell and fraction (perlin.h:72).
__device__ __forceinline__ float perlin2(int32_t ix, int32_t iy, float fx, float fy,
                                         uint32_t seed) {
    const uint32_t x0 = uint32_t(ix), y0 = uint32_t(iy);
    const uint32_t x1 = x0 + 1u, y1 = y0 + 1u;
    const float n00 = gradient2(corner2(x0, y0, seed), fx, fy);
    const float n10 = gradient2(corner2(x1, y0, seed), fx - 1.0f, fy);
    const float n01 = gradient2(corner2(x0, y1, seed), fx, fy - 1.0f);
    const float n11 = gradient2(corner2(x1, y1, seed), fx - 1.0f, fy - 1.0f);
    const float u = fade(fx);
    const float v = fade(fy);
    const float kSqrt2 = 1.41421356237309505f;
    return kSqrt2 * lerp(v, lerp(u, n00, n10), lerp(u, n01, n11));
}

// Lattice cell and fraction of a point (lattice.h:31).
struct Cell2 {
    int32_t ix, iy;
    float fx, fy;
};
__device__ __forceinline__ Cell2 split2(float x, float y) {
    const float cx = floorf(x);
    const float cy = floorf(y);
    return Cell2{int32_t(cx), int32_t(cy), x - cx, y - cy};
}

// Lattice cell and fraction of a double-precision point, the fraction taken before narrowing
// (lattice.h:49).
__device__ __forceinline__ Cell2 split2_precise(double x, double y) {
    const double cx = floor(x);
    const double cy = floor(y);
    return Cell2{int32_t(int64_t(cx)), int32_t(int64_t(cy)), float(x - cx), float(y - cy)};
}

__device__ __forceinline__ float perlin2(float x, float y, uint32_t seed) {
    const Cell2 c = split2(x, y);
    return perlin2(c.ix, c.iy, c.fx, c.fy, seed);
}

// --- simplex (simplex.h) ---------------------------------------------------------------------

__device__ __forceinline__ float simplex_corner(uint32_t ci, uint32_t cj, float dx, float dy,
                                                uint32_t seed) {
    const float t = 0.5f - dx * dx - dy * dy;
    const float t2 = t * t;
    const float c = t2 * t2 * gradient2(corner2(ci, cj, seed), dx, dy);
    return !(t <= 0.0f) ? c : 0.0f;
}

__device__ __forceinline__ float simplex2(float x, float y, uint32_t seed) {
    const float kSkew = 0.366025403784438647f;
    const float kUnskew = 0.211324865405187118f;
    const float skew = (x + y) * kSkew;
    const float cellX = floorf(x + skew);
    const float cellY = floorf(y + skew);
    const float unskew = (cellX + cellY) * kUnskew;
    const float x0 = x - (cellX - unskew);
    const float y0 = y - (cellY - unskew);
    const uint32_t stepX = x0 > y0 ? 1u : 0u;
    const uint32_t stepY = 1u - stepX;
    const float x1 = x0 - float(stepX) + kUnskew;
    const float y1 = y0 - float(stepY) + kUnskew;
    const float x2 = x0 - 1.0f + 2.0f * kUnskew;
    const float y2 = y0 - 1.0f + 2.0f * kUnskew;
    const uint32_t i = uint32_t(int32_t(cellX));
    const uint32_t j = uint32_t(int32_t(cellY));
    return 99.0f * (simplex_corner(i, j, x0, y0, seed) +
                    simplex_corner(i + stepX, j + stepY, x1, y1, seed) +
                    simplex_corner(i + 1u, j + 1u, x2, y2, seed));
}

// --- value (value.h) -------------------------------------------------------------------------

__device__ __forceinline__ float lattice_value(uint32_t x, uint32_t y, uint32_t seed) {
    return 2.0f * unit(pcg3d(U3{x, y, seed}).y) - 1.0f;
}

__device__ __forceinline__ float value2(float x, float y, uint32_t seed) {
    const Cell2 c = split2(x, y);
    const uint32_t x0 = uint32_t(c.ix), y0 = uint32_t(c.iy);
    const float v00 = lattice_value(x0, y0, seed);
    const float v10 = lattice_value(x0 + 1u, y0, seed);
    const float v01 = lattice_value(x0, y0 + 1u, seed);
    const float v11 = lattice_value(x0 + 1u, y0 + 1u, seed);
    const float u = fade(c.fx);
    const float v = fade(c.fy);
    return lerp(v, lerp(u, v00, v10), lerp(u, v01, v11));
}

// --- Worley (worley.h) -----------------------------------------------------------------------

struct WorleyD {
    float f1, f2, value;
};

__device__ __forceinline__ WorleyD worley2(float x, float y, uint32_t seed) {
    const Cell2 c = split2(x, y);
    float d1 = 1e30f, d2 = 1e30f;
    uint32_t nearest = 0u;
    for (int32_t dy = -2; dy <= 2; ++dy) {
        for (int32_t dx = -2; dx <= 2; ++dx) {
            const U3 h = pcg3d(U3{uint32_t(c.ix + dx), uint32_t(c.iy + dy), seed});
            const float px = float(dx) + unit(h.y) - c.fx;
            const float py = float(dy) + unit(h.z) - c.fy;
            const float d = px * px + py * py;
            if (d < d1) {
                d2 = d1;
                d1 = d;
                nearest = h.x;
            } else if (d < d2) {
                d2 = d;
            }
        }
    }
    return WorleyD{sqrtf(d1), sqrtf(d2), 2.0f * unit(nearest) - 1.0f};
}

// --- 3D Perlin, for the crater texture's radial streaks (perlin.h:40-60,113-128) -----------

__device__ __forceinline__ float gradient3(uint32_t hash, float x, float y, float z) {
    const uint32_t h = hash & 15u;
    const float u = h < 8u ? x : y;
    const float v = h < 4u ? y : (h == 12u || h == 14u ? x : z);
    return ((h & 1u) == 0u ? u : -u) + ((h & 2u) == 0u ? v : -v);
}

__device__ __forceinline__ float perlin3(float x, float y, float z, uint32_t seed) {
    const float cx = floorf(x), cy = floorf(y), cz = floorf(z);
    const uint32_t ix = uint32_t(int32_t(cx)), iy = uint32_t(int32_t(cy)),
                   iz = uint32_t(int32_t(cz));
    const float fx = x - cx, fy = y - cy, fz = z - cz;
    const uint32_t key = pcg(seed);
    float c[8];
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        const uint32_t dx = corner & 1u, dy = (corner >> 1u) & 1u, dz = corner >> 2u;
        const uint32_t h = pcg3d(U3{ix + dx, iy + dy, iz + dz + key}).x;
        c[corner] = gradient3(h, fx - float(dx), fy - float(dy), fz - float(dz));
    }
    const float u = fade(fx), v = fade(fy), w = fade(fz);
    const float near = lerp(v, lerp(u, c[0], c[1]), lerp(u, c[2], c[3]));
    const float far = lerp(v, lerp(u, c[4], c[5]), lerp(u, c[6], c[7]));
    return sclamp(lerp(w, near, far), -1.0f, 1.0f);
}

// One octave of any 2D basis, Worley distances mapped to [-1, 1] (fractal.h:91).
__device__ __forceinline__ float basis2(uint32_t basis, float x, float y, uint32_t seed) {
    const float kInvSqrt2 = 0.707106781186547524f;
    const float kInvSqrt5 = 0.447213595499957939f;
    switch (basis) {
    case kBasisSimplex:
        return simplex2(x, y, seed);
    case kBasisValue:
        return value2(x, y, seed);
    case kBasisWorleyF1:
        return 2.0f * smin(worley2(x, y, seed).f1 * kInvSqrt2, 1.0f) - 1.0f;
    case kBasisWorleyF2:
        return 2.0f * smin(worley2(x, y, seed).f2 * kInvSqrt5, 1.0f) - 1.0f;
    case kBasisWorleyF2MinusF1: {
        const WorleyD d = worley2(x, y, seed);
        return 2.0f * smin((d.f2 - d.f1) * kInvSqrt5, 1.0f) - 1.0f;
    }
    case kBasisVoronoi:
        return worley2(x, y, seed).value;
    default:
        return perlin2(x, y, seed);
    }
}

// --- fractals (fractal.h:146-262) ------------------------------------------------------------

// Golden-angle turn between successive octave lattices (fractal.h:146-148).
#define TGB_TURN_COS (-0.7373688780783197f)
#define TGB_TURN_SIN (0.6754902942615238f)

struct Sums {
    float weight, sum, total, feedback;
};

__device__ __forceinline__ Sums sums_start() {
    return Sums{1.0f, 0.0f, 0.0f, 1.0f};
}

// Adds one octave's signal to the running sums (fractal.h:169).
__device__ __forceinline__ Sums add_octave(Sums s, uint32_t type, float gain, float offset,
                                           int octave, float n) {
    switch (type) {
    case kTypeBillow:
        s.sum += s.weight * (2.0f * fabsf(n) - 1.0f);
        break;
    case kTypeRidged: {
        float signal = offset - fabsf(n);
        signal *= signal * s.feedback;
        s.feedback = sclamp(2.0f * signal, 0.0f, 1.0f);
        s.sum += s.weight * signal;
        break;
    }
    case kTypeHybrid: {
        const float signal = (n + offset) * s.weight;
        if (octave == 0) {
            s.sum = signal;
            s.feedback = signal;
        } else {
            s.feedback = sclamp(s.feedback, 0.0f, 1.0f);
            s.sum += s.feedback * signal;
            s.feedback *= signal;
        }
        break;
    }
    default:
        s.sum += s.weight * n;
        break;
    }
    s.total += s.weight;
    s.weight *= gain;
    return s;
}

// Normalised height from the sums over every octave (fractal.h:203).
__device__ __forceinline__ float finish(Sums s, uint32_t type, float amplitude, float offset) {
    switch (type) {
    case kTypeRidged: {
        const float ridge = smax(offset, 1.0f - offset);
        return amplitude * (2.0f * s.sum / (ridge * ridge * s.total) - 1.0f);
    }
    case kTypeHybrid:
        return amplitude * s.sum / ((1.0f + offset) * s.total);
    default:
        return amplitude * s.sum / s.total;
    }
}

// The octave seed and lattice offset of octave `o` of a fractal seeded `seed` (fractal.h:242).
struct Octave {
    uint32_t seed;
    float ox, oy;
};
__device__ __forceinline__ Octave octave_key(uint32_t seed, int o) {
    const U3 h = pcg3d(U3{seed, uint32_t(o), 0u});
    return Octave{h.x, unit(h.y), unit(h.z)};
}

// 2D fractal of any basis and type (fractal.h:219).
__device__ __forceinline__ float fractal2(float x, float y, const FractalParams& p) {
    float frequency = 1.0f / p.wavelength;
    float tc = 1.0f, ts = 0.0f;
    Sums s = sums_start();
    for (int o = 0; o < p.octaves; ++o) {
        const Octave k = octave_key(p.seed, o);
        const float rx = x * tc - y * ts;
        const float ry = x * ts + y * tc;
        const float n = basis2(p.basis, rx * frequency + k.ox, ry * frequency + k.oy, k.seed);
        s = add_octave(s, p.type, p.gain, p.offset, o, n);
        frequency *= p.lacunarity;
        const float nc = tc * TGB_TURN_COS - ts * TGB_TURN_SIN;
        ts = ts * TGB_TURN_COS + tc * TGB_TURN_SIN;
        tc = nc;
    }
    return finish(s, p.type, p.amplitude, p.offset);
}

// Golden-angle turn about (1, 2, 3) / sqrt(14) between 3D octave lattices (fractal.h:152-155).
__device__ __constant__ const float kTurn3[3][3] = {
    {-0.6132711010727254f, -0.293401570821183f, 0.7333580809050306f},
    {0.7897926788435601f, -0.24097777005594262f, 0.5640542870894418f},
    {0.011228581128535142f, 0.9251190369776896f, 0.37951111497202883f}};

// Perlin fBm in 3D, single precision, for kernels (fractal.h:247 `Fractal3Float`).
__device__ __forceinline__ float perlin_fbm3_float(float x, float y, float z, uint32_t seed,
                                                   int octaves, float gain) {
    float t[3][3] = {{1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}};
    float frequency = 1.0f;  // wavelength 1
    Sums s = sums_start();
    for (int o = 0; o < octaves; ++o) {
        const U3 h = pcg3d(U3{seed, uint32_t(o), 0u});
        const U3 g = pcg3d(U3{seed, uint32_t(o), 1u});
        const float rx = t[0][0] * x + t[0][1] * y + t[0][2] * z;
        const float ry = t[1][0] * x + t[1][1] * y + t[1][2] * z;
        const float rz = t[2][0] * x + t[2][1] * y + t[2][2] * z;
        const float n = perlin3(rx * frequency + unit(h.y), ry * frequency + unit(h.z),
                                rz * frequency + unit(g.x), h.x);
        s = add_octave(s, kTypeFbm, gain, 1.0f, o, n);
        frequency *= 2.0f;
        float next[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                next[r][c] = kTurn3[r][0] * t[0][c] + kTurn3[r][1] * t[1][c] + kTurn3[r][2] * t[2][c];
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                t[r][c] = next[r][c];
            }
        }
    }
    return finish(s, kTypeFbm, 1.0f, 1.0f);
}

// Perlin fBm specialisation of `fractal2`: the same operations in the same order, without the
// per-octave basis and type dispatch.
__device__ __forceinline__ float perlin_fbm2(float x, float y, uint32_t seed, float wavelength,
                                             float amplitude, int octaves, float lacunarity,
                                             float gain) {
    float frequency = 1.0f / wavelength;
    float tc = 1.0f, ts = 0.0f;
    float weight = 1.0f, sum = 0.0f, total = 0.0f;
    for (int o = 0; o < octaves; ++o) {
        const Octave k = octave_key(seed, o);
        const float rx = x * tc - y * ts;
        const float ry = x * ts + y * tc;
        const float n = perlin2(rx * frequency + k.ox, ry * frequency + k.oy, k.seed);
        sum += weight * n;
        total += weight;
        weight *= gain;
        frequency *= lacunarity;
        const float nc = tc * TGB_TURN_COS - ts * TGB_TURN_SIN;
        ts = ts * TGB_TURN_COS + tc * TGB_TURN_SIN;
        tc = nc;
    }
    return amplitude * sum / total;
}

__device__ __forceinline__ FractalParams params_of(const Fractal& f) {  // fractals.h:80
    return FractalParams{f.seed, f.wavelength, f.amplitude, f.octaves, f.lacunarity,
                         f.gain, f.basis, f.type, f.offset};
}

// Salt mixed into a fractal's seed for its warp fields (fractals.h:115).
#define TGB_WARP_SALT 0x5bd1e995u

// A fractal's value in [-1, 1], warped when it has a warp amplitude (fractals.h:151).
__device__ __forceinline__ float evaluate_fractal(float x, float y, const Fractal& f) {
    FractalParams unitp = params_of(f);
    unitp.amplitude = 1.0f;
    if (f.warpAmplitude > 0.0f) {
        FractalParams warp{pcg(f.seed ^ TGB_WARP_SALT), f.warpWavelength, f.warpAmplitude, 4, 2.0f,
                           0.5f, kBasisPerlin, kTypeFbm, 1.0f};
        const float dx = fractal2(x, y, warp);
        warp.seed = pcg(warp.seed);
        const float dy = fractal2(x, y, warp);
        return fractal2(x + dx, y + dy, unitp);
    }
    if (f.basis == kBasisPerlin && f.type == kTypeFbm) {
        return perlin_fbm2(x, y, f.seed, f.wavelength, 1.0f, f.octaves, f.lacunarity, f.gain);
    }
    return fractal2(x, y, unitp);
}

// Height of a stack of fractals: the first enabled one sets it, later ones blend
// (fractals.h:203-262).
__device__ __forceinline__ float evaluate_stack(float x, float y, const Fractal* fractals,
                                                uint32_t count) {
    float height = 0.0f;
    bool started = false;
    for (uint32_t i = 0; i < count; ++i) {
        const Fractal& f = fractals[i];
        if (!f.enabled) {
            continue;
        }
        const float value = evaluate_fractal(x, y, f);
        const float scaled = f.amplitude * value;
        if (!started) {
            height = scaled;
            started = true;
            continue;
        }
        switch (f.blend) {
        case kBlendMax:
            height = smax(height, scaled);
            break;
        case kBlendMin:
            height = smin(height, scaled);
            break;
        case kBlendMask:
            height *= 0.5f * (value + 1.0f);
            break;
        default:
            height += scaled;
            break;
        }
    }
    return height;
}

// --- 3D noise on a body (the reference runs it only on the CPU) ---------------------------------

// A lattice cell and fraction split in double precision (SplitLatticePrecise3, lattice.h:59).
struct Cell3 {
    int32_t ix, iy, iz;
    float fx, fy, fz;
};

__device__ __forceinline__ Cell3 split3_precise(double x, double y, double z) {
    const double cx = floor(x), cy = floor(y), cz = floor(z);
    return Cell3{int32_t(int64_t(cx)), int32_t(int64_t(cy)), int32_t(int64_t(cz)),
                 float(x - cx), float(y - cy), float(z - cz)};
}

// PerlinNoise3 at a cell (perlin.h:113-128): corner keys (x, y, z + pcg(seed)).
__device__ __forceinline__ float perlin3_cell(const Cell3& c, uint32_t seed) {
    const uint32_t key = pcg(seed);
    const uint32_t ix = uint32_t(c.ix), iy = uint32_t(c.iy), iz = uint32_t(c.iz);
    float k[8];
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        const uint32_t dx = corner & 1u, dy = (corner >> 1u) & 1u, dz = corner >> 2u;
        const uint32_t h = pcg3d(U3{ix + dx, iy + dy, iz + dz + key}).x;
        k[corner] = gradient3(h, c.fx - float(dx), c.fy - float(dy), c.fz - float(dz));
    }
    const float u = fade(c.fx), v = fade(c.fy), w = fade(c.fz);
    const float near = lerp(v, lerp(u, k[0], k[1]), lerp(u, k[2], k[3]));
    const float far = lerp(v, lerp(u, k[4], k[5]), lerp(u, k[6], k[7]));
    return sclamp(lerp(w, near, far), -1.0f, 1.0f);
}

// One corner of a 3D simplex (SimplexCorner3, simplex.h:27).
__device__ __forceinline__ float simplex_corner3(uint32_t ci, uint32_t cj, uint32_t ck, float dx,
                                                 float dy, float dz, uint32_t key) {
    const float t = 0.5f - dx * dx - dy * dy - dz * dz;
    if (t <= 0.0f) {
        return 0.0f;
    }
    const float t2 = t * t;
    return t2 * t2 * gradient3(pcg3d(U3{ci, cj, ck + key}).x, dx, dy, dz);
}

// SimplexNoise3 at a cell (simplex.h:72-115).
__device__ __forceinline__ float simplex3_cell(const Cell3& c, uint32_t seed) {
    const uint32_t key = pcg(seed);
    const int32_t cellSum = int32_t(uint32_t(c.ix) + uint32_t(c.iy) + uint32_t(c.iz));
    int32_t third = cellSum / 3;
    if (cellSum - 3 * third < 0) {
        third -= 1;
    }
    const float remainder = float(cellSum - 3 * third);
    const float skew = (remainder + c.fx + c.fy + c.fz) / 3.0f;
    const float stepX = floorf(c.fx + skew);
    const float stepY = floorf(c.fy + skew);
    const float stepZ = floorf(c.fz + skew);
    const float unskew = (remainder + stepX + stepY + stepZ) / 6.0f;
    const float x0 = c.fx - stepX + unskew;
    const float y0 = c.fy - stepY + unskew;
    const float z0 = c.fz - stepZ + unskew;
    const uint32_t i1 = x0 >= y0 && x0 >= z0 ? 1u : 0u;
    const uint32_t j1 = y0 > x0 && y0 >= z0 ? 1u : 0u;
    const uint32_t k1 = z0 > x0 && z0 > y0 ? 1u : 0u;
    const uint32_t i2 = x0 >= y0 || x0 >= z0 ? 1u : 0u;
    const uint32_t j2 = y0 > x0 || y0 >= z0 ? 1u : 0u;
    const uint32_t k2 = z0 > x0 || z0 > y0 ? 1u : 0u;
    const float kUnskew = 1.0f / 6.0f;
    const float x1 = x0 - float(i1) + kUnskew;
    const float y1 = y0 - float(j1) + kUnskew;
    const float z1 = z0 - float(k1) + kUnskew;
    const float x2 = x0 - float(i2) + 2.0f * kUnskew;
    const float y2 = y0 - float(j2) + 2.0f * kUnskew;
    const float z2 = z0 - float(k2) + 2.0f * kUnskew;
    const float x3 = x0 - 1.0f + 3.0f * kUnskew;
    const float y3 = y0 - 1.0f + 3.0f * kUnskew;
    const float z3 = z0 - 1.0f + 3.0f * kUnskew;
    const uint32_t i = uint32_t(c.ix) + uint32_t(third) + uint32_t(int32_t(stepX));
    const uint32_t j = uint32_t(c.iy) + uint32_t(third) + uint32_t(int32_t(stepY));
    const uint32_t k = uint32_t(c.iz) + uint32_t(third) + uint32_t(int32_t(stepZ));
    const float sum = simplex_corner3(i, j, k, x0, y0, z0, key) +
                      simplex_corner3(i + i1, j + j1, k + k1, x1, y1, z1, key) +
                      simplex_corner3(i + i2, j + j2, k + k2, x2, y2, z2, key) +
                      simplex_corner3(i + 1u, j + 1u, k + 1u, x3, y3, z3, key);
    return sclamp(76.0f * sum, -1.0f, 1.0f);
}

// ValueNoise3 at a cell (value.h:57-74): corner keys (x, y, z ^ pcg(seed)).
__device__ __forceinline__ float value3_cell(const Cell3& c, uint32_t seed) {
    const uint32_t key = pcg(seed);
    float v[8];
#pragma unroll
    for (uint32_t corner = 0; corner < 8u; ++corner) {
        const U3 at{uint32_t(c.ix) + (corner & 1u), uint32_t(c.iy) + ((corner >> 1u) & 1u),
                    (uint32_t(c.iz) + (corner >> 2u)) ^ key};
        v[corner] = 2.0f * unit(pcg3d(at).y) - 1.0f;
    }
    const float u = fade(c.fx), w = fade(c.fz), vv = fade(c.fy);
    const float near = lerp(vv, lerp(u, v[0], v[1]), lerp(u, v[2], v[3]));
    const float far = lerp(vv, lerp(u, v[4], v[5]), lerp(u, v[6], v[7]));
    return lerp(w, near, far);
}

// The squared gap from the fraction `f` to cell offset `d` (CellGapSquared, worley.h:24).
__device__ __forceinline__ float cell_gap2(int32_t d, float f) {
    float gap = 0.0f;
    if (d > 0) {
        gap = float(d) - f;
    } else if (d < 0) {
        gap = f - float(d + 1);
    }
    return gap * gap;
}

// Worley3 at a cell (worley.h:75-110): the 3 x 3 x 3 cells first, then the outer shell of the
// 5 x 5 x 5 where it can still hold the second nearest point; cell keys (x ^ pcg(seed), y, z).
__device__ __forceinline__ WorleyD worley3_cell(const Cell3& c, uint32_t seed) {
    const uint32_t seedKey = pcg(seed);
    float d1 = 1e30f, d2 = 1e30f;
    uint32_t nearest = 0u;
    for (int32_t shell = 0; shell < 2; ++shell) {
        for (int32_t dz = -2; dz <= 2; ++dz) {
            for (int32_t dy = -2; dy <= 2; ++dy) {
                for (int32_t dx = -2; dx <= 2; ++dx) {
                    const bool inner = abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1;
                    if (inner != (shell == 0)) {
                        continue;
                    }
                    if (shell == 1 &&
                        cell_gap2(dx, c.fx) + cell_gap2(dy, c.fy) + cell_gap2(dz, c.fz) >= d2) {
                        continue;
                    }
                    const U3 h = pcg3d(U3{uint32_t(c.ix + dx) ^ seedKey, uint32_t(c.iy + dy),
                                          uint32_t(c.iz + dz)});
                    const float px = float(dx) + unit(h.x) - c.fx;
                    const float py = float(dy) + unit(h.y) - c.fy;
                    const float pz = float(dz) + unit(h.z) - c.fz;
                    const float d = px * px + py * py + pz * pz;
                    if (d < d1) {
                        d2 = d1;
                        d1 = d;
                        nearest = pcg(h.x ^ h.y ^ h.z);
                    } else if (d < d2) {
                        d2 = d;
                    }
                }
            }
        }
    }
    return WorleyD{sqrtf(d1), sqrtf(d2), 2.0f * unit(nearest) - 1.0f};
}

// One octave of any 3D basis (BasisNoise3, fractal.h:115).
__device__ __forceinline__ float basis3(uint32_t basis, const Cell3& c, uint32_t seed) {
    const float kInvSqrt3 = 0.577350269189625765f;
    const float kInvSqrt6 = 0.408248290463863016f;
    switch (basis) {
    case kBasisSimplex:
        return simplex3_cell(c, seed);
    case kBasisValue:
        return value3_cell(c, seed);
    case kBasisWorleyF1:
        return 2.0f * smin(worley3_cell(c, seed).f1 * kInvSqrt3, 1.0f) - 1.0f;
    case kBasisWorleyF2:
        return 2.0f * smin(worley3_cell(c, seed).f2 * kInvSqrt6, 1.0f) - 1.0f;
    case kBasisWorleyF2MinusF1: {
        const WorleyD d = worley3_cell(c, seed);
        return 2.0f * smin((d.f2 - d.f1) * kInvSqrt6, 1.0f) - 1.0f;
    }
    case kBasisVoronoi:
        return worley3_cell(c, seed).value;
    default:
        return perlin3_cell(c, seed);
    }
}

// The golden-angle turn about (1, 2, 3) / sqrt(14) in double (Fractal3, fractal.h:286-289).
__device__ __constant__ const double kTurn3d[3][3] = {
    {-0.6132711010727254, -0.293401570821183, 0.7333580809050306},
    {0.7897926788435601, -0.24097777005594262, 0.5640542870894418},
    {0.011228581128535142, 0.9251190369776896, 0.37951111497202883}};

// Fractal3 (fractal.h:284-316): world coordinates in double, each octave's lattice point split
// in double before narrowing.
__device__ __forceinline__ float fractal3(double x, double y, double z, const FractalParams& p) {
    double frequency = 1.0 / double(p.wavelength);
    double t[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    Sums s = sums_start();
    for (int o = 0; o < p.octaves; ++o) {
        const U3 h = pcg3d(U3{p.seed, uint32_t(o), 0u});
        const U3 g = pcg3d(U3{p.seed, uint32_t(o), 1u});
        const double rx = t[0][0] * x + t[0][1] * y + t[0][2] * z;
        const double ry = t[1][0] * x + t[1][1] * y + t[1][2] * z;
        const double rz = t[2][0] * x + t[2][1] * y + t[2][2] * z;
        const double px = rx * frequency + double(unit(h.y));
        const double py = ry * frequency + double(unit(h.z));
        const double pz = rz * frequency + double(unit(g.x));
        const float n = basis3(p.basis, split3_precise(px, py, pz), h.x);
        s = add_octave(s, p.type, p.gain, p.offset, o, n);
        frequency *= double(p.lacunarity);
        double next[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                next[r][c] = kTurn3d[r][0] * t[0][c] + kTurn3d[r][1] * t[1][c] +
                             kTurn3d[r][2] * t[2][c];
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                t[r][c] = next[r][c];
            }
        }
    }
    return finish(s, p.type, p.amplitude, p.offset);
}

// EvaluateFractal3 with DomainWarp3 (fractals.h:218-243).
__device__ __forceinline__ float evaluate_fractal3(double x, double y, double z, const Fractal& f) {
    FractalParams unitp = params_of(f);
    unitp.amplitude = 1.0f;
    if (f.warpAmplitude > 0.0f) {
        FractalParams warp{pcg(f.seed ^ TGB_WARP_SALT), f.warpWavelength, f.warpAmplitude, 4, 2.0f,
                           0.5f, kBasisPerlin, kTypeFbm, 1.0f};
        const double dx = double(fractal3(x, y, z, warp));
        warp.seed = pcg(warp.seed);
        const double dy = double(fractal3(x, y, z, warp));
        warp.seed = pcg(warp.seed);
        const double dz = double(fractal3(x, y, z, warp));
        return fractal3(x + dx, y + dy, z + dz, unitp);
    }
    return fractal3(x, y, z, unitp);
}

// EvaluateFractals3 (fractals.h:262): the stack at a point of a body, blended as in 2D.
__device__ __forceinline__ float evaluate_stack3(double x, double y, double z,
                                                 const Fractal* fractals, uint32_t count) {
    float height = 0.0f;
    bool started = false;
    for (uint32_t i = 0; i < count; ++i) {
        const Fractal& f = fractals[i];
        if (!f.enabled) {
            continue;
        }
        const float value = evaluate_fractal3(x, y, z, f);
        const float scaled = f.amplitude * value;
        if (!started) {
            height = scaled;
            started = true;
            continue;
        }
        switch (f.blend) {
        case kBlendMax:
            height = smax(height, scaled);
            break;
        case kBlendMin:
            height = smin(height, scaled);
            break;
        case kBlendMask:
            height *= 0.5f * (value + 1.0f);
            break;
        default:
            height += scaled;
            break;
        }
    }
    return height;
}

}  // namespace noise
}  // namespace tgb
