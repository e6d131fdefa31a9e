/* tgb200 - a B200 (sm_100a) CUDA backend for TerrainGen's per-cell terrain evaluation path.
 *
 * The C ABI of libtgb200.so: plain pointers, sizes and status codes, no C++ or torch types. It is
 * the boundary the reference's GPU backend interface crosses today (src/gpu/kernel.h:46
 * `RunKernel`, src/gpu/device.h:49-68 `ComputeDevice`, `GpuDevice`), plus the hooks for the three
 * stages the reference runs only on the CPU (boulder baking, diamond-square refinement, the seam
 * solve). Each entry point names the reference interface it replaces.
 *
 * Parameter blocks are passed as the reference's own std430 bytes (`NoiseLayerKernel` 420 B,
 * `CraterShapeKernel` 188 B, `CraterRecord` 144 B each), exactly what its host code already
 * builds for RunKernel; sizes are checked.
 *
 * Memory: every compute entry point takes `memory`. With TG_MEMORY_HOST its buffers are host
 * memory, copied to the device and back inside the call, which returns when the result is in
 * place (RunKernel's contract). With TG_MEMORY_DEVICE they are device pointers and the work is
 * ordered on `stream` (a cudaStream_t; NULL for the device's own stream); the call may return
 * before the work finishes.
 *
 * Errors: a nonzero tg_status; tg_last_error() gives the message of the calling thread's last
 * failure. A device is thread-safe: calls on one device are serialized, as the reference's runs
 * are (src/gpu/cuda.cpp:303).
 */
#ifndef TGB200_H
#define TGB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TGB200_ABI_VERSION 1

typedef struct tg_device tg_device;

typedef enum tg_status {
    TG_OK = 0,
    TG_ERROR_ARGUMENT = 1,    /* a size, pointer or value is out of range */
    TG_ERROR_CUDA = 2,        /* the CUDA runtime failed; the message says how */
    TG_ERROR_UNSUPPORTED = 3, /* valid input this backend does not run (the caller's CPU path
                                 should take it, as RunKernel returning false asks) */
    TG_ERROR_MEMORY = 4,      /* a device allocation failed or a budget was exceeded */
    TG_ERROR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    TG_ERROR_STATE = 6        /* the call does not fit the object's state */
} tg_status;

enum { TG_MEMORY_HOST = 0, TG_MEMORY_DEVICE = 1 };

/* A north-up grid: the reference's GeoTransform coefficients in GDAL order
 * (include/terraingen/raster/geo_transform.h:17-35). Cell (col, row) is centered at
 * origin_x + (col + 0.5) * pixel_width, origin_y + (row + 0.5) * pixel_height. Rotated grids
 * (nonzero rotation terms) are TG_ERROR_UNSUPPORTED, as RunKernel refuses them
 * (src/gpu/kernel.cpp:44-48). Heights are row-major, row 0 first. */
typedef struct tg_grid {
    uint32_t width;
    uint32_t height;
    double origin_x;
    double pixel_width;
    double row_rotation;
    double origin_y;
    double col_rotation;
    double pixel_height;
} tg_grid;

/* No-data marking of a grid (src/gpu/kernel.cpp:28-31, Raster::NoData): mode 0 none, 1 NaN,
 * 2 `value`. Cells holding no-data are left as they are. */
typedef struct tg_nodata {
    uint32_t mode;
    float value;
} tg_nodata;

/* --- device ------------------------------------------------------------------------------- */

/* Opens CUDA device `ordinal` (replaces CudaCompute::Open / GpuDevice(Backend::Cuda),
 * src/gpu/cuda.cpp:188-240, src/gpu/device.h:68). Fails with TG_ERROR_UNSUPPORTED on a device
 * that is not sm_100. */
int tg_open(int ordinal, tg_device** device);
/* Releases the device's memory and stream. */
void tg_close(tg_device* device);
/* The message of the calling thread's last failure; "" when none. */
const char* tg_last_error(void);
/* ComputeDevice::DeviceName (src/gpu/device.h:41). */
int tg_device_name(tg_device* device, char* name, size_t capacity);
/* Waits for the device's stream. */
int tg_synchronize(tg_device* device);
/* How many times the binned crater and boulder kernels of this device poll a staged copy (a TMA
 * bulk copy into shared memory) before they give up on it and the call returns TG_ERROR_TIMEOUT
 * with the device still usable; by default 2^26 (seconds). 0 gives up without polling, which
 * exercises that error path without any fault. The reference has no counterpart: its CUDA
 * backend does not wait on device-side copies. */
int tg_set_wait_limit(tg_device* device, uint32_t polls);

/* --- noise (fBm sources and layers) --------------------------------------------------------- */

/* NoiseLayer on a grid: heights += the stacked fractals of the 420-byte `NoiseLayerKernel` at each
 * cell center measured from (origin_x, origin_y), cells holding no-data skipped. Replaces
 * RunKernel(backend, CompiledKernel<NoiseLayerKernel>(), kernel, grid, origin)
 * (src/layers/noise_layer.cpp:113-117; kernel src/layers/kernels/noise_layer.slang). Bit-exact
 * with the reference CPU path (AddNoiseRows, noise_layer.cpp:28). */
int tg_noise_layer(tg_device* device, const void* kernel, size_t kernel_bytes,
                   const tg_grid* grid, double origin_x, double origin_y, float* heights,
                   tg_nodata nodata, int memory, void* stream);

/* The same over RunKernel's strip buffers (src/gpu/kernel.cpp:98-111): per-column `xs` and
 * per-row `ys` positions, `rows` rows of `width` heights. */
int tg_noise_layer_rows(tg_device* device, const void* kernel, size_t kernel_bytes,
                        const float* xs, const float* ys, uint32_t width, uint32_t rows,
                        float* heights, tg_nodata nodata, int memory, void* stream);

/* SyntheticSource without posts on a grid: heights = elevation + the stacked `fractals` (`count`
 * 52-byte `Fractal`s, at most 8, disabled ones skipped) at each cell center. Replaces
 * SyntheticSource::FillSamples (src/sources/synthetic_source.cpp:87-95), which the reference runs
 * only on the CPU. Bit-exact with it. */
int tg_noise_source(tg_device* device, const void* fractals, uint32_t count, float elevation,
                    const tg_grid* grid, float* heights, int memory, void* stream);

/* SyntheticSource without posts on a sphere of `radius` meters: the grid is in degrees of
 * longitude (x) and latitude (y), and heights = elevation + the stacked `fractals` evaluated in 3D
 * at each cell center's position on the sphere (SyntheticSource::NoiseAt with FractalStackAt on a
 * body, src/noise/surface_noise.cpp:14-17: EvaluateFractals3 and Fractal3,
 * include/terraingen/noise/fractal.h:284, with lattice points split in double). The reference
 * runs this only on the CPU. Bit-exact with it: the cosines and sines of each column's longitude
 * and each row's latitude are taken on the host as the reference's UnitVector takes them. */
int tg_noise_source_body(tg_device* device, const void* fractals, uint32_t count,
                         float elevation, const tg_grid* grid, double radius, float* heights,
                         int memory, void* stream);

/* Conformance probe, the analogue of the reference's GPU test kernel
 * (tests/unit/gpu/kernels/noise_conformance.slang): for each of `n` points (x, y) in `xy`,
 * hashes[4i..4i+3] = PcgHash(i), Pcg3dHash(bits(x), bits(y), seed), and values[12i..12i+11] =
 * Perlin, simplex, value, Worley F1, F2, cell value, Perlin fBm / ridged / billow / hybrid
 * (wavelength 1000, amplitude 100, 8 octaves), 3D Perlin at (x, y, (x - y) / 2) and
 * Fractal3Float at (x, y, x / 4) with 3 octaves. */
int tg_noise_probe(tg_device* device, const float* xy, uint32_t n, uint32_t seed,
                   uint32_t* hashes, float* values, int memory);

/* --- craters ------------------------------------------------------------------------------ */

/* ApplyCraters' shaping on a plane grid: each cell holding data gets each crater of `records`
 * (`n` 144-byte `CraterRecord`s, with `data` their `n_data` variable-length floats) shaped by the
 * 188-byte `CraterShapeKernel`, at every cell of each 16x16 tile the crater's footprint touches,
 * as ShapeTilesOnCpu / ShapeTilesOnGpu do (src/layers/craters/shaping/apply.cpp:174-222). The
 * binning the reference does on the host (TileLists, apply.cpp:119) runs on the device.
 * `footprints` (optional; 3 doubles per crater: center x, y and reach in meters, as
 * CraterReach gives it) makes the footprint windows exactly the reference's; without it they
 * follow from the records. Craters with a datum are TG_ERROR_UNSUPPORTED here (their blend reads
 * the running height in apply order; tg_craters_apply_lists takes them), and the heights are left
 * as they were. Binning, scatter and shaping are ordered on the stream with no round trip to the
 * host; the call synchronizes once at the end to read its status. */
int tg_craters_apply(tg_device* device, const void* kernel, size_t kernel_bytes,
                     const void* records, uint32_t n, const float* data, uint32_t n_data,
                     const double* footprints, const tg_grid* grid, float* heights,
                     tg_nodata nodata, int memory, void* stream);

/* The drop-in strip form of the reference's crater kernel (src/layers/kernels/craters.slang,
 * bound by ShapeTilesOnGpu, apply.cpp:174-196): the host's tile lists `heads` (tiles across,
 * tile side, 0 for a plane, then first entry and count per tile) and `entries`, column
 * positions `xs` / `x_lows` [width] and row positions `ys` [rows] / `y_lows` [first_row + rows]
 * as MakeCellPositions builds them (apply.cpp:149-170). Craters apply in list order, datums
 * included. */
int tg_craters_apply_lists(tg_device* device, const void* kernel, size_t kernel_bytes,
                           const void* records, uint32_t n, const float* data, uint32_t n_data,
                           const uint32_t* heads, uint32_t n_heads, const uint32_t* entries,
                           uint32_t n_entries, const float* xs, const float* x_lows,
                           const float* ys, const float* y_lows, uint32_t width, uint32_t rows,
                           uint32_t first_row, float* heights, tg_nodata nodata, int memory,
                           void* stream);

/* The body form of the same kernel (craters.slang's branch for tiles[2] == 1: ShapeCratersOnBody,
 * include/terraingen/layers/kernels/craters.h:1360): `frames` holds the 52-byte CraterFrame of
 * each record, `points` the strip's cells as 24-byte SplitPoints (width x rows, positions on the
 * body, Surface::Position split), and each crater reads a cell in its frame (BodySplitOffset,
 * craters.h:208: the offset on the crater's tangent plane, azimuthal equidistant on a sphere).
 * Craters apply in list order, datums included. */
int tg_craters_apply_body(tg_device* device, const void* kernel, size_t kernel_bytes,
                          const void* records, uint32_t n, const float* data, uint32_t n_data,
                          const void* frames, const uint32_t* heads, uint32_t n_heads,
                          const uint32_t* entries, uint32_t n_entries, const void* points,
                          uint32_t width, uint32_t rows, uint32_t first_row, float* heights,
                          tg_nodata nodata, int memory, void* stream);


/* --- boulders ----------------------------------------------------------------------------- */

/* One boulder drawn as a dome: center (m), diameter (m), exposed height (m; Boulder::ExposedHeight,
 * include/terraingen/layers/boulders/boulder.h:84) and resolution weight (ResolutionWeight at the
 * spacing, src/layers/fade.cpp:50). 40 bytes. */
typedef struct tg_boulder {
    double x;
    double y;
    double diameter;
    double exposed_height;
    double weight;
} tg_boulder;

/* BoulderLayer's dome relief on a plane grid: every cell holding data within each boulder's box
 * (half-width 0.5 (diameter + width)) becomes max(height, base + weight * dome), base being the
 * cell's height before the call and the dome averaged over a band `width` meters wide (the
 * spacing; 0 samples it at the point). Replaces BoulderLayer::ApplySamples' DrawFeatures /
 * AddRelief / DomeHeight (src/layers/boulders/boulder_relief.cpp:44-57,244-275,426-439), which the
 * reference runs only on the CPU, for boulders without facets or fillets (the defaults). The
 * result does not depend on the boulders' order. */
int tg_boulders_bake(tg_device* device, const void* boulders, uint32_t n, double width,
                     const tg_grid* grid, float* heights, tg_nodata nodata, int memory,
                     void* stream);

/* tg_boulders_bake without any allocation, for callers that must not allocate GPU memory while
 * they evaluate: a streaming renderer's frame thread, where cudaMalloc or cudaFree would
 * synchronize the whole device and stall the frame, or a host that fixes its GPU memory at
 * start-up. No counterpart in the reference, which allocates per strip (src/gpu/cuda.cpp:244-313).
 * `boulders` (n tg_boulder) and `heights` are device memory; the work runs on `stream` (a
 * cudaStream_t; NULL for the legacy default stream) and the call returns when it is done. Its
 * scratch is one static 16 MiB device array inside the library, which every GPU that loads the
 * library holds until exit; at most 65536 boulders, 32768 bins of 32x32 cells (a 5792 x 5792 grid)
 * and 196608 binned boulders (TG_ERROR_MEMORY past that, found before anything is written, so the
 * heights are left as they were). The first call on a device finds the
 * array's device address (cudaGetSymbolAddress) and should come before any stream capture. Calls
 * share the array: calls whose work overlaps on the GPU race and must not overlap. Errors go to
 * `error` (capacity bytes, may be null), not to tg_last_error. */
int tg_boulders_bake_static(const void* boulders, uint32_t n, double width, const tg_grid* grid,
                            float* heights, tg_nodata nodata, void* stream, char* error,
                            size_t error_capacity);

/* --- diamond-square refinement ------------------------------------------------------------ */

/* DiamondSquareOptions (include/terraingen/sources/diamond_square.h:26-33) with a given scale:
 * fractal dimension D in [2, 3] (the displacement shrinks by 2^-((3 - D) / 2) per step), scale Se
 * (m), interp 0 bilinear or 1 Catmull-Rom (DiamondSquareInterp: Catmull-Rom midpoint means in
 * both steps and a Keys cubic read), seed, and min_pixel_size (m; 0 for none) capping the
 * levels. */
typedef struct tg_ds_options {
    double fractal_dimension;
    double scale;
    uint32_t interp;
    uint32_t seed;
    double min_pixel_size;
} tg_ds_options;

/* DiamondSquareUpsampler::FillSamples on a grid (src/sources/diamond_square.cpp:488-516), which
 * the reference runs only on the CPU: the `pw` x `ph` float posts on `post_grid` (row 0 north,
 * reads past the edge repeating it) refined Levels(post spacing, grid spacing) times and read
 * at every cell of `grid` into `heights`. Nodes are doubles; each block of output cells refines
 * the nodes it reads in on-chip memory, so only the heights are written to device memory. */
int tg_ds_refine(tg_device* device, const float* posts, uint32_t pw, uint32_t ph,
                 const tg_grid* post_grid, const tg_ds_options* options, const tg_grid* grid,
                 float* heights, int memory, void* stream);

/* tg_ds_refine on a window of a larger lattice of posts (a PostLattice read over a box:
 * src/sources/diamond_square.cpp:488-516 with Refinement::Frame at :302-309): `post_grid` is the
 * whole lattice's (its post (0, 0) anchors the node frame, so the displacement draws are the
 * lattice's own), and `posts` holds its columns [col0, col0 + pw) and rows [row0, row0 + ph),
 * reads past them repeating their edge. A window that ends at the lattice's bounds repeats its
 * edge as the reference's bounded lattices do; elsewhere the caller gives the window a margin of
 * posts beyond those the refinement reads (eight posts past the grid's bounds always suffice). */
int tg_ds_refine_window(tg_device* device, const float* posts, int64_t col0, int64_t row0,
                        uint32_t pw, uint32_t ph, const tg_grid* post_grid,
                        const tg_ds_options* options, const tg_grid* grid, float* heights,
                        int memory, void* stream);

/* Philox4x32-10 conformance (the analogue of the reference's Philox tests,
 * tests/unit/random/philox_test.cpp): for each of `n` sextets (counter x, y, z, w, key x, y) in
 * `in`, the four output words into `out`, and into `normals` the diamond-square displacement normal
 * of node (in[0], in[1]) as signed 32-bit indices at level in[2] & 31 with seed in[4]. Host
 * buffers. */
int tg_philox_probe(tg_device* device, const uint32_t* in, uint32_t n, uint32_t* out,
                    double* normals);

/* --- whole evaluations --------------------------------------------------------------------- */

/* A terrain as Terrain::Evaluate runs it on one grid (src/pipeline/terrain.cpp:289-331): a
 * synthetic source (`n_fractals` 52-byte Fractals plus `elevation`; none for a flat source at
 * `elevation`), then optionally a noise layer (a 420-byte NoiseLayerKernel, measured from the
 * origin), a crater layer (as tg_craters_apply takes it) and a boulder layer (as
 * tg_boulders_bake takes it), in that order. Every pointer is host memory for TG_MEMORY_HOST and
 * device memory for TG_MEMORY_DEVICE, like the heights. */
typedef struct tg_terrain {
    const void* fractals;
    uint32_t n_fractals;
    float elevation;
    const void* noise_layer;
    const void* crater_kernel;
    const void* crater_records;
    uint32_t n_craters;
    const float* crater_data;
    uint32_t n_crater_data;
    const double* crater_footprints;
    const void* boulders;
    uint32_t n_boulders;
    double boulder_width;
} tg_terrain;

/* Evaluates `terrain` on `grid` into `heights` (row-major, width x height floats): the source
 * fills, each layer applies in turn, all on the device; with host memory the layer inputs are
 * copied in once and the heights copied out once. Replaces Terrain::Evaluate / Fill for this
 * stack (src/pipeline/terrain.cpp:289-331). The call synchronizes once, at the end (the layers'
 * binning sizes itself on the device). On an error return the heights are unspecified. */
int tg_evaluate(tg_device* device, const tg_terrain* terrain, const tg_grid* grid,
                float* heights, int memory, void* stream);

/* Work counters of the device's last runs: counters[0] the (cell, crater) pairs the last crater
 * shaping evaluated, counters[1] the (cell, boulder) pairs the last boulder bake evaluated; at
 * most `n` are written. */
int tg_device_counters(tg_device* device, uint64_t* counters, size_t n);

/* The device's measured lane-operation rate for a mix of 32-bit integer multiply-adds and FP32
 * fused multiply-adds (the noise and shaping kernels' roofline denominator), in thread
 * instructions per second: dependent chains no compiler can shorten (quadratic IMAD, FFMA), so
 * the rate stays below the issue ceiling of 128 lanes per SM per clock. */
int tg_measure_alu(tg_device* device, double* lane_ops_per_second);

/* --- seams between chained sources ---------------------------------------------------------
 * A SourceChain fills an earlier source's gaps from a later source and joins the two
 * (ChainSeams, include/terraingen/sources/source_chain.h:24-62): the seam field is solved once on
 * the lattice of the earlier source's grid widened by the seam's reach (SeamLattice,
 * src/sources/source_chain.cpp:94) and read between its posts by Catmull-Rom interpolation. The
 * reference solves it on the CPU only (detail::BuildSeamField, src/sources/seam_field.cpp:663);
 * these replace it and FillGridGaps (source_chain.cpp:167). */

/* mode: 0 none, 1 feather, 2 height, 3 slope (ChainSeamMode). levels, sweeps and
 * coarsest_sweeps shape the multigrid preconditioner (4, 2 and 20 by default in the Python
 * layer); tolerance is the conjugate gradients' stop, relative to the first residual (1e-10 as
 * the reference when 0). */
typedef struct tg_seam_options {
    uint32_t mode;
    uint32_t levels;
    uint32_t sweeps;
    uint32_t coarsest_sweeps;
    double width;        /* Feather's band, in the lattice's units */
    double decay_length; /* L of Height and Slope; they reach 3 L beyond a gap's edge */
    double tolerance;
} tg_seam_options;

typedef struct tg_seam_stats {
    uint32_t unknowns;   /* posts solved for */
    uint32_t levels;     /* multigrid levels used */
    uint32_t iterations; /* conjugate gradient iterations */
    uint32_t reserved;
    double prepare_ms;   /* band, distances, unknowns and levels (device time) */
    double solve_ms;     /* the conjugate gradients (device time) */
} tg_seam_stats;

/* The seam field on a width x height lattice of posts dx by dy apart (row 0 first), from the
 * samples BuildSeamField starts from: `data` 1 where the earlier source has data, `difference` the
 * earlier source's height minus the later one's where both have data (NaN elsewhere). `field`
 * receives the correction at every post (0 where none). */
int tg_seam_solve(tg_device* device, const uint8_t* data, const float* difference,
                  uint32_t width, uint32_t height, double dx, double dy,
                  const tg_seam_options* options, float* field, int memory, void* stream);
/* What the calling thread's last tg_seam_solve did. */
int tg_seam_stats_get(tg_seam_stats* stats);
/* FillGridGaps: each cell of `heights` (on `grid`) holding no data takes `later` (the later
 * source's height on the same grid) plus the field (posts on `lattice`) read at the cell's
 * center by Catmull-Rom interpolation; cells where `later` has no data are left alone.
 * `window` (host memory, may be null for the whole grid) limits the cells visited to
 * col0, row0, width, height: the later source's window, outside which it has no data. */
int tg_seam_fill(tg_device* device, const float* field, const tg_grid* lattice,
                 const float* later, const tg_grid* grid, float* heights, tg_nodata nodata,
                 const uint32_t* window, int memory, void* stream);
/* SampleSources (seam_field.cpp:76-113) for two sources held as rasters on one grid: the lattice
 * is the `lw` x `lh` posts whose first post is cell (`col0`, `row0`) of `grid` (negative, or past
 * the grid's edge, where the lattice pads it; its posts there have no data). `data` gets 1 where
 * `earlier` has data (finite, and not the no-data value), `difference` earlier minus later (in
 * double, rounded to float) where both have, NaN elsewhere. */
int tg_seam_samples(tg_device* device, const float* earlier, const float* later,
                    const tg_grid* grid, int64_t col0, int64_t row0, uint32_t lw, uint32_t lh,
                    tg_nodata nodata, uint8_t* data, float* difference, int memory,
                    void* stream);

/* Crater datums: the relief of the older craters under each fitted crater's datum footprint
 * (KernelDatumRelief, include/terraingen/layers/kernels/craters.h:1214-1316), which RunKernel runs
 * for FitDatumsWithKernel (src/layers/craters/shaping/datum_fit.cpp:303-328) with the program
 * src/layers/kernels/crater_datums.slang. `kernel` is the 200-byte CraterDatumKernel, read on
 * the host in either memory mode (a parameter block, as tg_craters_apply's); records
 * (144 bytes each), data, the band floats and cells, cells, entries and targets are the index the
 * reference builds (IndexDatumRelief, datum_fit.cpp:268-296). `heights` is the lattice strip:
 * `rows` rows of `width` points (one row per fitted crater, from target `first_row`), each point
 * receiving its relief added. */
int tg_crater_datums(tg_device* device, const void* kernel, size_t kernel_bytes,
                     const void* records, uint32_t n_records, const float* data, uint32_t n_data,
                     const float* band_floats, uint32_t n_band_floats, const uint32_t* band_cells,
                     uint32_t n_band_cells, const uint32_t* cells, uint32_t n_cells,
                     const uint32_t* entries, uint32_t n_entries, const uint32_t* targets,
                     uint32_t n_targets, uint32_t width, uint32_t rows, uint32_t first_row,
                     float* heights, int memory, void* stream);

/* The body form (src/layers/kernels/crater_body_datums.slang, bound by FitBodyDatumsOnGpu,
 * src/layers/craters/shaping/datum_fit.cpp): each lattice point of a strip (`positions`, 24-byte
 * SplitPoints, width x rows) gets the relief of the craters its row lists (`lists`: per row its
 * first entry and count into `entries`), each crater read in its 52-byte CraterFrame within its
 * `bounds` (KernelBodyDatumRelief, include/terraingen/layers/kernels/craters.h:1326); `kernel` is
 * the 188-byte CraterBodyDatumKernel; points holding `nodata` are left as they are. */
int tg_crater_body_datums(tg_device* device, const void* kernel, size_t kernel_bytes,
                          const void* records, uint32_t n_records, const float* data,
                          uint32_t n_data, const void* frames, const float* bounds,
                          const uint32_t* lists, uint32_t n_lists, const uint32_t* entries,
                          uint32_t n_entries, const void* positions, uint32_t width,
                          uint32_t rows, uint32_t first_row, float* heights, tg_nodata nodata,
                          int memory, void* stream);

/* --- crater populations and kernel batches (host) ------------------------------------------ */

/* A crater layer's population on a plane: a power-law density N(>D) = c D^-exponent per m^2 on
 * [min_diameter, max_diameter] (PowerLawSfd, include/terraingen/distribution/power_law.h:54),
 * uniform ages over lifetime_gyr (UniformAges, ages/age_model.h:46), constant fresh depth and rim
 * ratios worn by FreshnessDegradation (degradation/freshness_degradation.h:22), seeded by `seed`
 * (CraterLayerOptions::seed). */
typedef struct tg_crater_population {
    uint32_t seed;
    double sfd_coefficient;
    double sfd_exponent;
    double min_diameter;
    double max_diameter;
    double lifetime_gyr;
    double depth_ratio;
    double rim_ratio;
    double cutoff_depth_ratio;    /* kVisibilityDepthRatio, 0.04 */
    double cell_size_factor;      /* CraterGenerationOptions::cellSizeFactor, 16 */
    double margin_radii;          /* candidate margin in radii (tg_crater_population only) */
    double min_resolved_diameter; /* bands wholly below are skipped (tg_crater_population only) */
} tg_crater_population;

/* How the layer shapes its craters.
 * `profile`: 0 Fassett-Thomson, 1 Martin-Parkes-Dunstan, 2 and 3 a ComplexCraterProfile over
 *   those (include/terraingen/layers/craters/profiles/complex.h:78) with the lunar shape
 *   (LunarComplexCraterShape, src/layers/craters/shaping/morphometry.cpp:40) from
 *   `transition_diameter` meters: flat floors, central peaks, a power-law exterior to 3 radii.
 * `irregular`: 1 for DefaultCraterApply (apply_options.cpp:49): irregular outlines, wall
 *   terraces (CraterTerraces) and massif central peaks (CraterPeaks) at their defaults; 0 for
 *   plain CraterApplyOptions (none of them).
 * Terraces: with `terrace_onset` > 0 the three terrace fields replace CraterTerraces'
 *   onsetDiameter, fullDiameter and minFreshness (apply_options.h:183-226); otherwise the
 *   defaults (20 km, 65 km, 0.3). */
typedef struct tg_crater_shaping {
    uint32_t profile;
    uint32_t irregular;
    double transition_diameter;
    double terrace_onset;
    double terrace_full;
    double terrace_min_freshness;
} tg_crater_shaping;

/* Host threads tg_crater_batch and tg_boulder_generate use (0, the default, for every core), as
 * EvaluationOptions::threads sets the reference's (include/terraingen/pipeline/terrain.h). The
 * results do not depend on it: work is split by generation rows and crater blocks and joined in
 * order. */
void tg_set_host_threads(unsigned threads);

/* The craters the layer draws over `region` (x0, y0, x1, y1 in meters), in the reference's order
 * (GenerateCraters, src/layers/craters/generation/population.cpp:414): centers, diameters, ages
 * and 64-bit ids, bit-exact. `count` receives the number; arrays (any may be null) hold at most
 * `capacity`. Host only. */
int tg_crater_generate(const tg_crater_population* population, const double* region,
                       double* x, double* y, double* diameter, double* age, uint64_t* id,
                       size_t capacity, size_t* count);

/* tg_crater_generate on the device: one thread per generation cell of every band, the kept
 * craters in the reference's order into `x`, `y`, `diameter`, `age` and `id` (device pointers
 * with TG_MEMORY_DEVICE, host pointers with TG_MEMORY_HOST; at most `capacity`; `count` receives
 * the number). Every per-band constant comes from the host's libm; the device's `pow` (the
 * diameter's inversion), `log` and `lgamma` (PTRS's acceptance) remain, so diameters may differ
 * from tg_crater_generate's in their last bits while counts, positions, ages and ids match. A cell
 * whose Poisson acceptance or keep decision lies within `tolerance` (relative; 0 for 1e-9) of its
 * threshold is drawn on the host instead. Replaces GenerateCraters' cell loop
 * (src/layers/craters/generation/population.cpp:381-441), which the reference runs on the CPU. */
int tg_crater_generate_device(tg_device* device, const tg_crater_population* population,
                              const double* region, double* x, double* y, double* diameter,
                              double* age, uint64_t* id, size_t capacity, size_t* count,
                              double tolerance, int memory, void* stream);

/* A boulder layer's sizes and pose (BoulderLayerOptions, include/terraingen/layers/boulders/
 * boulder_options.h): power-law sizes N(>D) = c D^-exponent per m^2 on [min_diameter,
 * max_diameter] (BoulderSizes with a PowerLawSfd), height ratio and buried share uniform between
 * their bounds (BoulderPose), the resolution fade in samples (ResolutionFade, 2 and 4), and the
 * candidate cells' size factor (16). */
typedef struct tg_boulder_population {
    uint32_t seed;
    double sfd_coefficient;
    double sfd_exponent;
    double min_diameter;
    double max_diameter;
    double min_height_ratio;
    double max_height_ratio;
    double min_burial;
    double max_burial;
    double fade_start_samples;
    double fade_end_samples;
    double cell_size_factor;
} tg_boulder_population;

/* The boulders a BoulderLayer with these sizes and pose, and otherwise its defaults (no patches,
 * clusters, density or slope maps, crater ejecta, bedrock, fragmentation, settling or facets, on
 * a plane), draws into a grid of `spacing` over `region` (x0, y0, x1, y1 in meters; the reference
 * bakes over the grid's bounds grown by half a sample): PlaceBoulders (src/layers/boulders/
 * boulder_layer.cpp:263-405) restated, bit-exact, in the reference's order, as the 40-byte
 * tg_boulder tg_boulders_bake takes (x, y, diameter, exposed height, resolution weight), those
 * of positive weight only. `count` receives the number; `out` (may be null) holds at most
 * `capacity`. Host only. */
int tg_boulder_generate(const tg_boulder_population* population, const double* region,
                        double spacing, tg_boulder* out, size_t capacity, size_t* count);

/* What CraterLayer::ApplySamples hands the crater kernel for `grid`
 * (src/layers/craters/crater_layer.cpp:337-359, shaping/apply.cpp:339-370): the 188-byte
 * CraterShapeKernel, the 144-byte CraterRecords of the craters on the grid in apply order, their
 * float data, and 3 doubles per record (center x, y and footprint reach) for tg_craters_apply.
 * Call with null outputs to learn `n_records` and `n_data`. Host only. */
int tg_crater_batch(const tg_crater_population* population, const tg_crater_shaping* shaping,
                    const tg_grid* grid, void* kernel, void* records, size_t record_capacity,
                    float* data, size_t data_capacity, double* footprints, size_t* n_records,
                    size_t* n_data);

/* tg_crater_batch with the apply order and the records made on the device: the population and
 * the wall terraces and massif peaks of the craters that carry them are made on the host threads
 * as tg_crater_batch makes them, the apply order by stable radix sorts on the device, then one
 * device thread per crater draws its outline, takes its footprint and writes its record, data
 * floats and footprint; `records`, `data` and `footprints`
 * are device memory (any may be null; all null asks for the sizes), `kernel` host memory. The
 * outputs are tg_crater_batch's byte for byte. Ordered on `stream` (the device's own when null);
 * the call synchronizes it once, to read the sizes; `staged_bytes` (may be null) receives the bytes
 * it copied to the device (64 per candidate crater, 4 per terrace or peak float). Replaces
 * the same host work as tg_crater_batch
 * (MakeCraterKernelBatch, src/layers/craters/shaping/crater_kernel.cpp:187-622, after
 * PrepareCraters, src/layers/craters/shaping/prepared.cpp:60). TG_ERROR_ARGUMENT, the sizes set,
 * when a capacity is below them (no output written past it). */
int tg_crater_batch_device(tg_device* device, const tg_crater_population* population,
                           const tg_crater_shaping* shaping, const tg_grid* grid, void* kernel,
                           void* records, size_t record_capacity, float* data,
                           size_t data_capacity, double* footprints, size_t* n_records,
                           size_t* n_data, size_t* staged_bytes, void* stream);

/* --- output -------------------------------------------------------------------------------- */

/* GeoTiffWriteOptions (include/terraingen/raster/geotiff/geotiff.h:185): compression in
 * TiffCompression's order (0 None, 1 LZW, 3 Deflate; 2, PackBits, is refused as the reference
 * refuses it), tile_size a positive multiple of 16 (256 in the reference), big_tiff 1 to always
 * write BigTIFF (otherwise only when the tiles could pass 4 GiB). */
typedef struct tg_geotiff_options {
    uint32_t compression;
    uint32_t tile_size;
    uint32_t big_tiff;
    uint32_t reserved;
} tg_geotiff_options;

/* GeoKeys (geotiff.h:31): the GeoKeyDirectory, GeoDoubleParams and GeoAsciiParams tags' values;
 * no keys when directory_count is 0. */
typedef struct tg_geokeys {
    const uint16_t* directory;
    uint32_t directory_count;
    uint32_t double_count;
    const double* double_params;
    const char* ascii_params; /* NUL-terminated, or null */
} tg_geokeys;

/* WriteGeoTiff (src/raster/geotiff/geotiff_write.cpp:256-297): `band_count` float rasters of
 * grid->width x grid->height cells (row 0 first) on `grid`'s transform, as a tiled little-endian
 * float32 GeoTIFF at `path`; `nodata` (mode 1 NaN, 2 value) is the GDAL_NODATA tag and pads the
 * edge tiles (0 without). The tiles are laid out, run through the floating-point predictor and,
 * for LZW, compressed on the device; Deflate tiles are compressed on host threads with zlib
 * (level 6, the reference's miniz level: the same decoded data, other bytes). With None or LZW
 * the file is the reference's byte for byte. `bands` are device pointers with
 * TG_MEMORY_DEVICE (read on `stream`), host pointers with TG_MEMORY_HOST. */
int tg_geotiff_write(tg_device* device, const char* path, const float* const* bands,
                     uint32_t band_count, const tg_grid* grid, tg_nodata nodata,
                     const tg_geokeys* keys, const tg_geotiff_options* options, int memory,
                     void* stream);

/* --- batched tiles ---------------------------------------------------------------------------
 * Many tiles of one layer stack (a Perlin fBm source, a crater layer and a boulder layer)
 * evaluated together: one count / scan / scatter of every tile's craters and boulders into bins,
 * then ONE persistent launch in which each CTA takes bins from a device work queue and writes
 * each cell once (source, craters, boulders). The launches are captured in two CUDA graphs
 * (binning, evaluation) on the first evaluation and replayed while the batch fits the plan's
 * capacities. World-to-lattice
 * offsets are split in double per tile and octave, so tiles far from the origin keep float
 * lattice fractions (heights within 1e-3 m of an FP64 evaluation at 1.7e6 m). The reference
 * evaluates tiles one at a time (Terrain::EvaluateTiles, src/pipeline/terrain.cpp:158); this is
 * its batched form. */
typedef struct tg_batch tg_batch;

/* One tile of a batch. Cell (col, row) of the tile is heights[height_offset + row * pitch + col].
 * Its craters are records [crater_begin, crater_begin + crater_count) of the batch, their data
 * offsets relative to crater_data + data_begin (what tg_crater_batch returns for the tile's grid);
 * its boulders are [boulder_begin, boulder_begin + boulder_count), baked with dome band width
 * `boulder_width` (the tile's sample spacing). */
typedef struct tg_tile {
    tg_grid grid;
    uint64_t height_offset;
    uint32_t pitch;
    uint32_t crater_begin;
    uint32_t crater_count;
    uint32_t data_begin;
    uint32_t boulder_begin;
    uint32_t boulder_count;
    double boulder_width;
} tg_tile;

/* One set of scattered point queries of a batch (Terrain::EvaluatePoints,
 * src/pipeline/terrain.cpp:133): points [point_begin, point_begin + point_count) of the batch's
 * `points` (x, y doubles), point i's height going to heights[height_offset + i]. Craters and
 * boulders as a tile's; a crater or boulder changes a point within its reach. */
typedef struct tg_point_set {
    uint32_t point_begin;
    uint32_t point_count;
    uint64_t height_offset;
    uint32_t crater_begin;
    uint32_t crater_count;
    uint32_t data_begin;
    uint32_t boulder_begin;
    uint32_t boulder_count;
    uint32_t reserved;
    double boulder_width;
} tg_point_set;

/* A batch's inputs (host memory). `fractals` holds `n_fractals` 52-byte Fractals of which at most
 * one is enabled, a Perlin fBm without warp; `crater_kernel` is one CraterShapeKernel for every
 * tile; crater_footprints (optional) holds 3 doubles per record as tg_crater_batch writes them.
 * Tiles and point sets may name the same records and boulders. */
typedef struct tg_batch_input {
    const tg_tile* tiles;
    uint32_t n_tiles;
    const void* fractals;
    uint32_t n_fractals;
    float elevation;
    const void* crater_kernel;
    const void* crater_records;
    uint32_t n_craters;
    const float* crater_data;
    uint32_t n_crater_data;
    const double* crater_footprints;
    const tg_boulder* boulders;
    uint32_t n_boulders;
    const tg_point_set* point_sets;
    uint32_t n_point_sets;
    const double* points;
    uint32_t n_points;
} tg_batch_input;

/* What the batch last did. */
typedef struct tg_batch_stats {
    uint32_t variant;            /* kernel shape in use (tg_batch_variant) */
    uint32_t bin_width, bin_height, cells_per_thread;
    uint32_t fast;               /* 1: the lean crater path */
    uint32_t bins;               /* bins (work items) of the loaded batch */
    uint64_t cells;              /* cells of the loaded batch */
    uint64_t crater_pairs;       /* (cell, crater) pairs the last evaluation shaped */
    uint64_t boulder_pairs;      /* (cell, boulder) pairs it baked */
    uint64_t crater_entries;     /* binned entries */
    uint64_t boulder_entries;
    uint32_t captures;           /* CUDA graphs captured so far */
    uint32_t replays;            /* graph launches so far */
    float bin_ms;                /* device time of the last binning (count, scan, scatter) */
    float evaluate_ms;           /* device time of the last persistent evaluation */
    float graph_ms;              /* device time of the last binning + evaluation, end to end */
    uint32_t ctas;               /* persistent CTAs of the last evaluation */
} tg_batch_stats;

int tg_batch_create(tg_device* device, tg_batch** batch);
void tg_batch_destroy(tg_batch* batch);
/* Copies `input` to the device and plans capacities (the next evaluation re-captures its graph
 * when they grow). Fails with TG_ERROR_UNSUPPORTED for a source other than one unwarped Perlin
 * fBm, for rotated tile grids and for crater datums. */
int tg_batch_load(tg_batch* batch, const tg_batch_input* input);
/* Evaluates the loaded batch into `heights` (n_heights floats; device pointer for
 * TG_MEMORY_DEVICE, else host memory the result is copied to). Stream-ordered on `stream` in
 * device mode; returns after the evaluation has finished. */
int tg_batch_evaluate(tg_batch* batch, float* heights, size_t n_heights, int memory,
                      void* stream);
/* tg_batch_load then tg_batch_evaluate. */
int tg_batch_run(tg_batch* batch, const tg_batch_input* input, float* heights, size_t n_heights,
                 int memory, void* stream);
/* The autotuner: evaluates the loaded batch with every kernel shape (bin size, cells per thread),
 * `trials` timed replays each after a warm-up, and keeps the fastest. `ms` (optional) receives
 * each variant's median time, tg_batch_variant_count() values. */
int tg_batch_tune(tg_batch* batch, int trials, float* ms);
int tg_batch_variant_count(void);
/* Selects a kernel shape by index (0 .. tg_batch_variant_count() - 1); bin_width, bin_height and
 * cells_per_thread (optional) describe it. */
int tg_batch_set_variant(tg_batch* batch, int index);
int tg_batch_variant(int index, uint32_t* bin_width, uint32_t* bin_height,
                     uint32_t* cells_per_thread);
int tg_batch_stats_get(tg_batch* batch, tg_batch_stats* stats);

/* --- serving -----------------------------------------------------------------------------------
 * A request server for the streaming-renderer use case: tile and point-query requests are
 * submitted as they arrive and evaluated by continuous batching. Whenever one of the server's
 * batch slots is free, the requests waiting then (up to max_batch_cells, and within the device
 * memory budget) become one batch, launched on the slot's own stream while earlier batches may
 * still run; tg_server_poll hands back the finished requests. Crater records are built per
 * feature region (a square of region_cells cells of a level of detail, owning the craters whose
 * centers lie in it) and kept resident in device memory, least recently used regions evicted
 * first. Each request's heights are the same whichever requests share its batch. The reference
 * evaluates such requests one at a time (Terrain::EvaluateTiles / EvaluatePoints,
 * src/pipeline/terrain.cpp:133-158); this form has no counterpart there. */
typedef struct tg_server tg_server;

typedef struct tg_server_options {
    const void* fractals;           /* the source: at most one enabled Perlin fBm Fractal */
    uint32_t n_fractals;
    float elevation;
    tg_crater_population craters;   /* the crater layer */
    tg_crater_shaping shaping;
    double base_spacing;            /* finest level of detail, meters; levels are base * 2^k */
    double point_spacing;           /* the level whose craters point queries take */
    uint64_t hbm_budget;            /* device bytes the server may hold */
    uint64_t max_batch_cells;       /* cells admitted into one batch (at least one request) */
    uint32_t slots;                 /* batches in flight, 1 to 8 */
    uint32_t region_cells;          /* side of a feature region in cells of its level */
    int32_t variant;                /* batch kernel shape; -1 lets the autotuner pick */
    uint32_t reserved;
    /* The DEM-refinement stack (DiamondSquareUpsampler over a DEM, src/sources/diamond_square.cpp:
     * 488-516): with post_spacing > 0 the source is the fBm above sampled at a post lattice of
     * that spacing (post (i, j) at (i * post_spacing, -j * post_spacing), rounded to float as a
     * DEM's posts) and refined by diamond-square under `refine` to each tile's spacing (point
     * queries: point_spacing), the craters added on top; 0 evaluates the fBm at every cell. */
    double post_spacing;
    tg_ds_options refine;
} tg_server_options;

typedef struct tg_request {
    uint64_t id;
    uint32_t kind;                  /* 0 a tile, 1 a set of points */
    uint32_t memory;                /* where `heights` lies: TG_MEMORY_HOST or TG_MEMORY_DEVICE */
    tg_grid grid;                   /* tile: north up, spacing base_spacing * 2^k */
    const double* points;           /* points: n_points (x, y) pairs (host), copied at submit */
    uint32_t n_points;
    float* heights;                 /* where the heights go (row-major tile, or one per point),
                                       valid until the request is handed back; device heights are
                                       written by a device-to-device copy on the server's stream */
} tg_request;

typedef struct tg_server_stats {
    uint64_t submitted, completed, batches, cells;
    uint64_t regions_built, regions_evicted, regions_resident;
    uint64_t feature_bytes;         /* device bytes reserved for resident regions */
    uint64_t device_bytes;          /* device bytes the server holds now */
    uint64_t peak_bytes;            /* most it has held */
    uint64_t deferred;              /* admissions put off by the memory budget */
    double gpu_ms;                  /* device time of the batches (binning + evaluation) */
    double region_ms;               /* host time spent building regions */
} tg_server_stats;

int tg_server_create(tg_device* device, const tg_server_options* options, tg_server** server);
void tg_server_destroy(tg_server* server);
/* Queues a request (TG_ERROR_ARGUMENT for a malformed one). */
int tg_server_submit(tg_server* server, const tg_request* request);
/* Advances the server: hands back finished batches' requests (their heights written) and launches
 * waiting requests into free slots. `ids` receives up to `capacity` finished request ids and
 * `count` how many; with `wait` set it blocks until at least one request finishes while any is
 * queued or running. */
int tg_server_poll(tg_server* server, int wait, uint64_t* ids, size_t capacity, size_t* count);
int tg_server_stats_get(tg_server* server, tg_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* TGB200_H */
