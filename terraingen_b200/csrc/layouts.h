// Byte layouts of the parameter blocks TerrainGen's evaluation path hands to a GPU backend.
//
// These mirror, field for field, the std430 structs the reference uploads through
// RunKernel (src/gpu/kernel.h:46): the bytes a caller passes through the C ABI are the bytes the
// reference's host code already builds, so nothing is re-packed at the boundary. Each struct names
// the reference declaration it mirrors and asserts its size as the reference does.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define TG_HD __host__ __device__
#else
#define TG_HD
#endif

namespace tgb {

// --- noise (include/terraingen/noise/fractals.h:58-75, fractal.h:21-43) -------------------------

enum : uint32_t { kBasisPerlin = 0, kBasisSimplex = 1, kBasisValue = 2, kBasisWorleyF1 = 3,
                  kBasisWorleyF2 = 4, kBasisWorleyF2MinusF1 = 5, kBasisVoronoi = 6 };
enum : uint32_t { kTypeFbm = 0, kTypeRidged = 1, kTypeBillow = 2, kTypeHybrid = 3 };
enum : uint32_t { kBlendAdd = 0, kBlendMax = 1, kBlendMin = 2, kBlendMask = 3 };

// `Fractal` (fractals.h:58). The reference's first member is a C++ `bool`: one byte, then three
// bytes of padding whose contents are unspecified, so only the first byte is read.
struct Fractal {
    uint8_t enabled;
    uint8_t pad_[3];
    uint32_t seed;
    float wavelength;
    float amplitude;
    int32_t octaves;
    float lacunarity;
    float gain;
    uint32_t basis;
    uint32_t type;
    float offset;
    uint32_t blend;
    float warpAmplitude;
    float warpWavelength;
};
static_assert(sizeof(Fractal) == 52, "Fractal must match its std430 layout");

constexpr uint32_t kMaxFractals = 8;  // fractals.h:45

// `NoiseLayerKernel` / `FractalStack` (noise_layer.h:19, fractals.h:95).
struct FractalStack {
    Fractal fractals[kMaxFractals];
    uint32_t count;
};
static_assert(sizeof(FractalStack) == 420, "NoiseLayerKernel must match its std430 layout");

// `FractalParams` (fractal.h:53): what one fractal's octave loop reads.
struct FractalParams {
    uint32_t seed;
    float wavelength;
    float amplitude;
    int32_t octaves;
    float lacunarity;
    float gain;
    uint32_t basis;
    uint32_t type;
    float offset;
};

// --- craters (include/terraingen/layers/kernels/craters.h:26-139) ------------------------------

enum : uint32_t { kProfileFassettThomson = 0, kProfileMartinParkesDunstan = 1,
                  kProfileTabulated = 2 };

struct CraterProfileKernel {  // craters.h:26
    uint32_t simple;
    uint32_t rim;
    uint32_t complex;
    uint32_t diffused;
    float transitionDiameter;
    float floorCoefficient;
    float floorExponent;
    float peakHeightCoefficient;
    float peakHeightExponent;
    float peakWidthCoefficient;
    float peakWidthExponent;
    uint32_t peakFromVolume;
    float peakFitMaxDiameter;
    float ejectaExponent;
    float complexReachRadii;
    float tableExtent;
    uint32_t tableCells;
    uint32_t agesOffset;
    uint32_t ageCount;
};
static_assert(sizeof(CraterProfileKernel) == 76, "CraterProfileKernel must match std430");

struct CraterShapeKernel {  // craters.h:49
    CraterProfileKernel profile;
    float reachRadii;
    float profileReachRadii;
    float blendStart;
    float blendEnd;
    uint32_t blendShape;
    float interiorReplacement;
    float replaceStart;
    float replaceEnd;
    float mantling;
    float ejectaReachRadii;
    float rimSigma;
    float rimInner;
    float rimOuter;
    float rimStrength;
    uint32_t rimShape;
    float noiseAmplitude;
    float noiseWavelength;
    int32_t noiseOctaves;
    float noiseGain;
    float noiseRimAmplitude;
    float noiseRimWavelength;
    float noiseRimInner;
    float noiseRimOuter;
    float wallStreaks;
    float wallStreakWidth;
    float ejecta;
    float ejectaLineation;
    float minFreshness;
};
static_assert(sizeof(CraterShapeKernel) == 188, "CraterShapeKernel must match std430");

// What fitting crater datums takes (craters.h:1214): the craters' shapes, the fit footprint in
// radii, the lattice points per side across it, and the size bands of the crater index.
struct CraterDatumKernel {
    CraterShapeKernel shape;
    float fitRadii;
    uint32_t latticeSide;
    uint32_t bandCount;
};
static_assert(sizeof(CraterDatumKernel) == 200, "CraterDatumKernel must match std430");

struct CraterRecord {  // craters.h:81
    float x;
    float y;
    float diameter;
    float resolution;
    float freshDepth;
    float freshRim;
    float currentDepth;
    float currentRim;
    float diffusion;
    float ellipticity;
    float heading;
    uint32_t firstHarmonic;
    uint32_t harmonicCount;
    uint32_t harmonicOffset;
    uint32_t tableCount;
    uint32_t tableOffset;
    uint32_t profileOffset;
    uint32_t hasDatum;
    float datumA;
    float datumB;
    float datumC;
    uint32_t noiseKey;
    uint32_t textureKey;
    uint32_t markCount;
    uint32_t markOffset;
    float shiftX;
    float shiftY;
    float upslopeX;
    float upslopeY;
    uint32_t terraceCount;
    uint32_t terraceOffset;
    uint32_t peakCount;
    uint32_t peakOffset;
    uint32_t replace;
    float xLow;
    float yLow;
};
static_assert(sizeof(CraterRecord) == 144, "CraterRecord must match std430");

struct CraterFrame {  // craters.h:128
    float x, y, z;
    float eastX, eastY, eastZ;
    float northX, northY, northZ;
    float sphereRadius;
    float xLow, yLow, zLow;
};
static_assert(sizeof(CraterFrame) == 52, "CraterFrame must match std430");

struct SplitPoint {  // craters.h:186
    float x, xLow, y, yLow, z, zLow;
};

}  // namespace tgb
