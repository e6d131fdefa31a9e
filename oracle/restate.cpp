// oracle/restate.cpp - test infrastructure only (see restate.h). Build: make -C oracle restate.
// Compiled with -ffp-contract=off so the float forms round as the reference's build does.
#include "restate.h"

#include <algorithm>
#include <cmath>

namespace {

// Octave lattice turn (fractal.h:146-148), as floats and as the doubles they came from.
const float kTurnCosF = -0.7373688780783197f;
const float kTurnSinF = 0.6754902942615238f;

template <typename T> T Fade(T t) {  // lattice.h:79
    return t * t * t * (t * (t * T(6) - T(15)) + T(10));
}

template <typename T> T Lerp(T t, T a, T b) {  // lattice.h:84
    return a + t * (b - a);
}

template <typename T> T Gradient(uint32_t hash, T x, T y) {  // perlin.h:17
    const uint32_t h = hash & 7u;
    const T inv = T(0.707106781186547524);
    const T axis = (h & 2u) ? y : x;
    const T sx = h == 5u ? -x : x;
    const T sy = h == 6u ? -y : y;
    const T sum = sx + sy;
    const T diag = (h == 7u ? -sum : sum) * inv;
    return h < 4u ? ((h & 1u) ? -axis : axis) : diag;
}

uint32_t Corner(uint32_t x, uint32_t y, uint32_t seed) {
    uint32_t out[3];
    rs_pcg3d(x, y, seed, out);
    return out[0];
}

template <typename T> T Perlin(int32_t ix, int32_t iy, T fx, T fy, uint32_t seed) {  // perlin.h:72
    const uint32_t x0 = uint32_t(ix), y0 = uint32_t(iy);
    const T one = T(1);
    const T n00 = Gradient<T>(Corner(x0, y0, seed), fx, fy);
    const T n10 = Gradient<T>(Corner(x0 + 1u, y0, seed), fx - one, fy);
    const T n01 = Gradient<T>(Corner(x0, y0 + 1u, seed), fx, fy - one);
    const T n11 = Gradient<T>(Corner(x0 + 1u, y0 + 1u, seed), fx - one, fy - one);
    const T u = Fade(fx), v = Fade(fy);
    return T(1.41421356237309505) * Lerp(v, Lerp(u, n00, n10), Lerp(u, n01, n11));
}

template <typename T> T PerlinAt(T x, T y, uint32_t seed) {
    const T cx = std::floor(x), cy = std::floor(y);
    return Perlin<T>(int32_t(int64_t(cx)), int32_t(int64_t(cy)), x - cx, y - cy, seed);
}

float HashUnit(uint32_t h) {  // hash.h:60
    return float(h >> 8u) * 0x1p-24f;
}

}  // namespace

extern "C" {

uint32_t rs_pcg(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

void rs_pcg3d(uint32_t x, uint32_t y, uint32_t z, uint32_t* out) {
    x = x * 1664525u + 1013904223u;
    y = y * 1664525u + 1013904223u;
    z = z * 1664525u + 1013904223u;
    x += y * z;
    y += z * x;
    z += x * y;
    x ^= x >> 16u;
    y ^= y >> 16u;
    z ^= z >> 16u;
    x += y * z;
    y += z * x;
    z += x * y;
    out[0] = x;
    out[1] = y;
    out[2] = z;
}

float rs_perlin2_f32(float x, float y, uint32_t seed) {
    return PerlinAt<float>(x, y, seed);
}

double rs_perlin2_f64(double x, double y, uint32_t seed) {
    return PerlinAt<double>(x, y, seed);
}

float rs_fbm2_f32(float x, float y, uint32_t seed, float wavelength, float amplitude, int octaves,
                  float lacunarity, float gain) {
    float frequency = 1.0f / wavelength;
    float tc = 1.0f, ts = 0.0f;
    float weight = 1.0f, sum = 0.0f, total = 0.0f;
    for (int o = 0; o < octaves; ++o) {
        uint32_t h[3];
        rs_pcg3d(seed, uint32_t(o), 0u, h);
        const float rx = x * tc - y * ts;
        const float ry = x * ts + y * tc;
        const float n = rs_perlin2_f32(rx * frequency + HashUnit(h[1]),
                                       ry * frequency + HashUnit(h[2]), h[0]);
        sum += weight * n;
        total += weight;
        weight *= gain;
        frequency *= lacunarity;
        const float nc = tc * kTurnCosF - ts * kTurnSinF;
        ts = ts * kTurnCosF + tc * kTurnSinF;
        tc = nc;
    }
    return amplitude * sum / total;
}

double rs_fbm2_f64(double x, double y, uint32_t seed, double wavelength, double amplitude,
                   int octaves, double lacunarity, double gain) {
    // The same lattice (the turn's float constants, the hashed offsets) with double arithmetic.
    double frequency = 1.0 / wavelength;
    double tc = 1.0, ts = 0.0;
    double weight = 1.0, sum = 0.0, total = 0.0;
    for (int o = 0; o < octaves; ++o) {
        uint32_t h[3];
        rs_pcg3d(seed, uint32_t(o), 0u, h);
        const double rx = x * tc - y * ts;
        const double ry = x * ts + y * tc;
        const double n = rs_perlin2_f64(rx * frequency + double(HashUnit(h[1])),
                                        ry * frequency + double(HashUnit(h[2])), h[0]);
        sum += weight * n;
        total += weight;
        weight *= gain;
        frequency *= lacunarity;
        const double c = double(kTurnCosF), s = double(kTurnSinF);
        const double nc = tc * c - ts * s;
        ts = ts * c + tc * s;
        tc = nc;
    }
    return amplitude * sum / total;
}

void rs_fbm_grid_f32(uint32_t width, uint32_t height, double x0, double y0, double pixel,
                     uint32_t seed, float wavelength, float amplitude, int octaves,
                     float lacunarity, float gain, float elevation, float* out) {
    for (uint32_t r = 0; r < height; ++r) {
        const float y = float(y0 + (double(r) + 0.5) * -pixel);
        for (uint32_t c = 0; c < width; ++c) {
            const float x = float(x0 + (double(c) + 0.5) * pixel);
            // EvaluateFractals: amplitude * unit fBm; the source adds its elevation.
            out[size_t(r) * width + c] =
                elevation +
                amplitude * rs_fbm2_f32(x, y, seed, wavelength, 1.0f, octaves, lacunarity, gain);
        }
    }
}

void rs_fbm_grid_f64(uint32_t width, uint32_t height, double x0, double y0, double pixel,
                     uint32_t seed, double wavelength, double amplitude, int octaves,
                     double lacunarity, double gain, double elevation, double* out) {
    for (uint32_t r = 0; r < height; ++r) {
        const double y = y0 + (double(r) + 0.5) * -pixel;
        for (uint32_t c = 0; c < width; ++c) {
            const double x = x0 + (double(c) + 0.5) * pixel;
            out[size_t(r) * width + c] =
                elevation + rs_fbm2_f64(x, y, seed, wavelength, amplitude, octaves, lacunarity, gain);
        }
    }
}

double rs_crater_profile_f64(int profile, uint32_t rim, double distance, double diameter,
                             double freshDepth, double freshRim, double currentDepth,
                             double currentRim) {
    const double radius = 0.5 * diameter;
    if (profile == 1) {  // Martin, Parkes and Dunstan (craters.h:389)
        const double depth = currentDepth * diameter, rimH = currentRim * diameter;
        const double fresh = freshRim * diameter;
        const double x = distance / radius - 1.0;
        if (x >= 1.0) {
            return 0.0;
        }
        const double k = fresh - rimH + depth;
        const double alpha = (rimH - fresh) / k;
        if (x <= alpha) {
            return (k * x + 2.0 * k) * x + fresh;
        }
        if (x <= 0.0) {
            return k * (alpha + 1.0) / alpha * x * x + rimH;
        }
        const double scale0 = 0.14 * std::pow(radius, 0.74);
        const double es = fresh > 0.0 ? scale0 * rimH / fresh : scale0;
        auto exterior = [&](double t, double& slope) {
            const double offset = rimH - es;
            const double gradient = -es / 8.0 - offset;
            const double r = 1.0 / (t + 1.0);
            const double law = es * r * r * r + offset + gradient * t;
            const double lawSlope = -3.0 * es * r * r * r * r + gradient;
            const double taper = 1.0 - t * t;
            slope = lawSlope * taper - 2.0 * t * law;
            return law * taper;
        };
        const double beta = std::min(1.0, 1.5 * (fresh - rimH) / k);
        if (x <= beta) {
            double joinSlope;
            const double join = exterior(beta, joinSlope);
            const double drop = rimH - join;
            const double slope = drop > 0.0 ? std::max(joinSlope, -3.0 * drop / beta) : joinSlope;
            const double t = x / beta;
            return rimH + (join - rimH) * t * t * (3.0 - 2.0 * t) + beta * slope * t * t * (t - 1.0);
        }
        double unused;
        return exterior(x, unused);
    }
    // Fassett and Thomson (craters.h:338), over the diameter.
    const double x = distance / radius;
    if (x > 1.5) {
        return 0.0;
    }
    auto exterior = [](double t, double start) {
        const double p = 0.188253307 + t * (-0.187050452 + t * (0.01844746 + t * 0.01505647));
        const double u = (t - start) / (1.5 - start);
        return p * (1.0 - u * u);
    };
    const double interior = -0.228809953 + x * (0.227533882 + x * (0.083116795 - x * 0.039499407));
    double h;
    if (rim == 2u) {
        h = x <= 0.98 ? interior : (x <= 1.02 ? freshRim : exterior(x, 1.02));
    } else {
        const double edge = rim == 0u ? 0.98 : 1.0;
        h = x <= 0.2 ? -0.181 : (x <= edge ? interior : exterior(x, edge));
    }
    return std::max(h, freshRim - currentDepth) * diameter;
}

void rs_philox(const uint32_t* counter, const uint32_t* key, uint32_t* out) {
    uint32_t c[4] = {counter[0], counter[1], counter[2], counter[3]};
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = uint64_t(0xD2511F53u) * c[0];
        const uint64_t p1 = uint64_t(0xCD9E8D57u) * c[2];
        const uint32_t n[4] = {uint32_t(p1 >> 32) ^ c[1] ^ k0, uint32_t(p1),
                               uint32_t(p0 >> 32) ^ c[3] ^ k1, uint32_t(p0)};
        for (int i = 0; i < 4; ++i) {
            c[i] = n[i];
        }
    }
    for (int i = 0; i < 4; ++i) {
        out[i] = c[i];
    }
}

double rs_ds_normal(int64_t col, int64_t row, int level, uint32_t seed) {
    const uint32_t counter[4] = {uint32_t(col), uint32_t(row),
                                 uint32_t(level) | (uint32_t((col >> 32) ^ (row >> 32)) << 5), 0u};
    const uint32_t key[2] = {seed, 0x524D4450u};
    uint32_t w[4];
    rs_philox(counter, key, w);
    const double u1 = double((uint64_t(w[0] >> 5u) << 26u) | uint64_t(w[1] >> 6u)) * 0x1p-53;
    const double u2 = double((uint64_t(w[2] >> 5u) << 26u) | uint64_t(w[3] >> 6u)) * 0x1p-53;
    return std::sqrt(-2.0 * std::log1p(-u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
}

}  // extern "C"
