/* oracle/restate.h - test infrastructure only, never linked into the product.
 *
 * A CPU restatement of the reference's per-cell evaluation math, written from the reference's
 * formulas, in two precisions: `_f32` functions follow the reference's float arithmetic step by
 * step (built with -ffp-contract=off, so they reproduce its golden vectors bit for bit), `_f64`
 * functions evaluate the same formulas in double with the same integer lattice hashes: the FP64
 * oracle heights are reported against.
 *
 * Pinned against the reference's own golden vectors (tests/golden/noise/kernels_test.cpp) and the
 * reference CPU path built from its sources (oracle/_ref/libtgref.so); see tests/test_oracle.py.
 */
#ifndef TG_RESTATE_H
#define TG_RESTATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint32_t rs_pcg(uint32_t v);                                   /* hash.h:33 */
void rs_pcg3d(uint32_t x, uint32_t y, uint32_t z, uint32_t* out); /* hash.h:40 */
float rs_perlin2_f32(float x, float y, uint32_t seed);         /* perlin.h:106 */
double rs_perlin2_f64(double x, double y, uint32_t seed);

/* Perlin fBm Fractal2 (fractal.h:219) with the reference's parameter order. */
float rs_fbm2_f32(float x, float y, uint32_t seed, float wavelength, float amplitude, int octaves,
                  float lacunarity, float gain);
double rs_fbm2_f64(double x, double y, uint32_t seed, double wavelength, double amplitude,
                   int octaves, double lacunarity, double gain);

/* A grid of Perlin fBm heights (elevation + fbm) at the cell centers of a north-up grid, the
 * SyntheticSource fill: f32 narrows positions to float as the reference does, f64 keeps them. */
void rs_fbm_grid_f32(uint32_t width, uint32_t height, double x0, double y0, double pixel,
                     uint32_t seed, float wavelength, float amplitude, int octaves,
                     float lacunarity, float gain, float elevation, float* out);
void rs_fbm_grid_f64(uint32_t width, uint32_t height, double x0, double y0, double pixel,
                     uint32_t seed, double wavelength, double amplitude, int octaves,
                     double lacunarity, double gain, double elevation, double* out);

/* Round simple craters in FP64 (no outline, rim smoothing, noise, texture, terraces or peaks):
 * Fassett-Thomson (profile 0, rim mode `rim`) or Martin-Parkes-Dunstan (profile 1) heights of
 * crater state (fresh depth/rim, current depth/rim ratios) at `distance` from a crater of
 * `diameter` (craters.h:338-421). */
double rs_crater_profile_f64(int profile, uint32_t rim, double distance, double diameter,
                             double freshDepth, double freshRim, double currentDepth,
                             double currentRim);

/* Philox4x32-10 (include/terraingen/random/philox.h:82) of `counter` and `key` into `out`. */
void rs_philox(const uint32_t* counter, const uint32_t* key, uint32_t* out);
/* The standard normal diamond-square draws for node (col, row) of `level` with `seed`:
 * RandomStream(seed, kMidpointDisplacementStream, col, row, level | high << 5) then
 * StandardNormal (src/sources/diamond_square.cpp:382, src/random/samplers.cpp:65). */
double rs_ds_normal(int64_t col, int64_t row, int level, uint32_t seed);

#ifdef __cplusplus
}
#endif

#endif
