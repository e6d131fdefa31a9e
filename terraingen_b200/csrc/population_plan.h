// The per-band plan of a crater population (GenerateCraters on a plane, no spacing, density map
// or manual craters: src/layers/craters/generation/population.cpp): what the device generator
// needs from the host, every constant computed with the host libm as the reference computes it,
// and the host's own cell generation for the cells the device hands back.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/tgb200.h"

namespace tgb {
namespace host {

struct CraterBandPlan {
    uint32_t exponent;                      // the band's k: diameters in [2^k, 2^(k+1))
    double low, high, cellSize;
    int32_t iMin, jMin, iMax, jMax;         // its cells
    double mean;                            // expected craters per cell
    // SamplePoisson's constants (samplers.cpp:14-55): the multiplication limit exp(-mean) below
    // 10, PTRS's above it.
    double limit, sqrtMean, logMean, b, a, inverseAlpha, vr, logInverseAlpha;
    // PowerLawSfd::Sample (power_law.h): N(lo) - N(hi), N(lo), -1 / e.
    double count, top, inverseExponent;
    double inner[4], outer[4];              // the keep boxes (x0, y0, x1, y1)
    uint64_t firstCell;                     // cells of the bands before
};

struct HostCrater {
    double x, y, diameter, age;
    uint64_t id;
};

std::vector<CraterBandPlan> crater_plan(const tg_crater_population& spec, const double* region);

// The kept craters of cell (i, j) of `band`, in draw order, on the host.
void cell_kept(const tg_crater_population& spec, const double* region,
               const CraterBandPlan& band, int32_t i, int32_t j, std::vector<HostCrater>& out);

}  // namespace host
}  // namespace tgb
