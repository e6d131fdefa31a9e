// Launchers of the device kernels, called by the C ABI (api.cu). Every launcher is
// stream-ordered, takes device pointers only and returns the launch's cudaError_t.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "layouts.h"

namespace tgb {

// A non-rotated grid's GeoTransform (include/terraingen/raster/geo_transform.h:17-35): cell
// (col, row) has its center at originX + (col + 0.5) * pixelWidth + (row + 0.5) * rowRotation,
// originY + (col + 0.5) * colRotation + (row + 0.5) * pixelHeight.
struct Grid {
    uint32_t width, height;
    double originX, pixelWidth, rowRotation, originY, colRotation, pixelHeight;
};

// How no-data cells are marked (src/gpu/kernel.cpp:28-31): none, NaN, or a value.
struct NoData {
    uint32_t mode;
    float value;
};

// Where a kernel reads cell positions: computed from the grid in double and narrowed after
// subtracting `originX/Y` (what RunKernel's xs/ys hold, src/gpu/kernel.cpp:56-71), or read from
// per-column and per-row arrays when given.
struct Positions {
    double originX, originY;
    const float* xs;  // optional, [width]
    const float* ys;  // optional, [height]
};

// --- noise ---------------------------------------------------------------------------------
// heights[row * width + col] = base + stack(x, y), where base is `elevation` when `fill` is set
// and the cell's current height otherwise (cells holding no-data are skipped then).
cudaError_t launch_noise(const FractalStack& stack, const Grid& grid, const Positions& at,
                         bool fill, float elevation, NoData nodata, float* heights,
                         cudaStream_t stream);

// Conformance probe (the reference's tests/unit/gpu/kernels/noise_conformance.slang analogue):
// for each input point, the PCG hashes and basis/fractal values, for testing against the oracle.
// A SyntheticSource on a sphere: `lons` / `lats` hold (cos, sin) of each column's longitude and
// each row's latitude.
cudaError_t launch_noise_body(const FractalStack& stack, float elevation, uint32_t width,
                              uint32_t height, const double* lons, const double* lats,
                              double radius, float* heights, cudaStream_t stream);

cudaError_t launch_noise_probe(const float* xy, uint32_t n, uint32_t seed, uint32_t* hashes,
                               float* values, cudaStream_t stream);

// --- craters -------------------------------------------------------------------------------
// Side of the square bins craters are sorted into for shaping, in cells.
constexpr uint32_t kBinCells = 32;
// Side of the reference's crater tiles (src/layers/craters/shaping/apply.cpp:109); a crater is
// evaluated at every cell of each such tile its footprint window touches.
constexpr uint32_t kRefTileCells = 16;

// One crater binned for shaping: its record, the inclusive range of reference tiles its
// footprint touches, and the distance (m) beyond which no cell can be within its reach (+inf
// when marks, terraces or a floor shift leave no such bound). 160 bytes, so a bin's entries copy
// to shared memory in 16-byte units.
struct BinEntry {
    CraterRecord record;
    uint16_t tileX0, tileX1, tileY0, tileY1;
    float cull;
    uint32_t index;
};
static_assert(sizeof(BinEntry) == 160, "BinEntry must be a multiple of 16 bytes");

struct CraterBins {
    uint32_t binsX, binsY;
    uint32_t* counts;    // [bins + 1]: entries per bin, then exclusive offsets after the scan
    uint32_t* cursor;    // [bins]
    BinEntry* entries;   // [capacity]
    uint32_t capacity;
    uint32_t* total;     // [1] entries needed
    int4* boxes;         // [craters] reference-tile box per crater (x0, x1, y0, y1); empty: x0 > x1
    float* culls;        // [craters] cull distance per crater
    uint32_t firstBin;   // the bin of a launch's first block (a strip of bin rows)
    uint32_t* pairStart; // [craters + 1]: bins per crater, then their exclusive scan
    uint32_t* extrasMark;  // [bins], zeroed: a bin listed for the extras pass
    uint32_t* extrasList;  // [bins + 1], [0] zeroed: how many bins are listed, then the bins
};

// Per crater: its footprint's reference-tile box on `grid` and the number of bins it covers,
// added to bins.counts. `footprints` (x, y, reach in meters, as doubles) is optional; without it
// the footprint follows from the record (center hi + lo, reach = outline stretch x reachRadii x
// radius).
// `scratch` holds scan_scratch_words(n) words for the scan of the pairs.
cudaError_t launch_crater_count(const CraterShapeKernel& k, const CraterRecord* records,
                                uint32_t n, const float* data, const double* footprints,
                                const Grid& grid, const CraterBins& bins, uint32_t* scratch,
                                cudaStream_t stream);
// The plain path's lean craters (crater_math.cuh LeanCrater): kLeanCraterBytes per crater, made
// by launch_crater_lean; with them the bins hold kLeanEntryBytes entries, else 160-byte BinEntry.
// The plain path's lean craters (crater_math.cuh LeanCrater): kLeanCraterBytes per crater, made
// by launch_crater_lean after the count pass (it reads the footprint boxes and culls). With them
// the bins hold 4-byte crater indices (the shaping kernel gathers each entry's LeanCrater into
// shared memory), else 160-byte BinEntry copies of the records.
constexpr size_t kLeanCraterBytes = 208;
constexpr size_t kLeanEntryBytes = 4;
cudaError_t launch_crater_lean(const CraterShapeKernel& k, const CraterRecord* records, uint32_t n,
                               const float* data, const CraterBins& bins, void* leans,
                               cudaStream_t stream);
// Scatters each crater into its bins (its index when `leans` is given, else a BinEntry); an entry
// whose crater needs the extras pass (crater_needs_extras) carries kHeavyEntry in its index.
cudaError_t launch_crater_scatter(const CraterShapeKernel& k, const CraterRecord* records,
                                  uint32_t n, const Grid& grid, const CraterBins& bins,
                                  const void* leans, cudaStream_t stream);
constexpr uint32_t kHeavyEntry = 0x80000000u;
// Whether a batch takes the lean shaping path (crater_math.cuh `fast_contribution`): the
// kernel's options allow it and the count pass saw no record feature beyond outlines
// (`batchFlags` bit 2). The batched and served forms use this whole-batch rule.
bool crater_fast_path(const CraterShapeKernel& k, uint32_t batchFlags);
// Whether the plain path's binned kernel shapes the batch lean entry by entry: the kernel's
// options allow the lean path (a closed-form simple profile, complex craters allowed, no rim
// smoothing, noise or texture); entries marked kHeavyEntry (complex craters, terraces, peaks,
// tables, marks, shifts) take the general path inside the same launch.
bool crater_lean_entries(const CraterShapeKernel& k);
// The lean path's harmonics: (amplitude cos phase, amplitude sin phase) at the data's offsets.
cudaError_t launch_crater_harmonics(const CraterRecord* records, uint32_t n, const float* data,
                                    float* harmonics, cudaStream_t stream);
// Polls of a staged copy before a binned kernel gives up on it (flag 2, TG_ERROR_TIMEOUT).
constexpr uint32_t kWaitPolls = 1u << 26;

// Shapes the bins of rows [firstBinRow, firstBinRow + binRows): with `leans` (index bins) the lean
// kernel, then, when `extras`, the extras pass over the same bins; otherwise the general kernel on
// BinEntry bins.
cudaError_t launch_crater_shape(const CraterShapeKernel& k, const CraterRecord* records,
                                const float* data, const void* leans, bool extras,
                                const Grid& grid,
                                NoData nodata, const CraterBins& bins, float* heights,
                                cudaStream_t stream, uint32_t firstBinRow = 0,
                                uint32_t binRows = 0xffffffffu, uint32_t polls = kWaitPolls);

// The drop-in form: the reference's own tile lists (`CraterTiles`, apply.cpp:111-143), craters
// applied in list order exactly as ShapeTilesOnCpu does (apply.cpp:199-222).
cudaError_t launch_crater_shape_lists(const CraterShapeKernel& k, const CraterRecord* records,
                                      const float* data, const uint32_t* heads,
                                      const uint32_t* entries, uint32_t width, uint32_t rows,
                                      uint32_t firstRow, const float* xs, const float* xLows,
                                      const float* ys, const float* yLows, NoData nodata,
                                      float* heights, cudaStream_t stream);

// The body form: each cell's position a split point in 3D, each crater read in its frame.
cudaError_t launch_crater_shape_body(const CraterShapeKernel& k, const CraterRecord* records,
                                     const CraterFrame* frames, const float* data,
                                     const uint32_t* heads, const uint32_t* entries,
                                     uint32_t width, uint32_t rows, uint32_t firstRow,
                                     const SplitPoint* points, const NoData& nodata,
                                     float* heights, cudaStream_t stream);

// --- boulders ------------------------------------------------------------------------------
// One boulder drawn as a dome (tg_boulder in include/tgb200.h).
struct BoulderRecord {
    double x, y, diameter, exposedHeight, weight;
};
static_assert(sizeof(BoulderRecord) == 40, "BoulderRecord is 5 doubles");

// A boulder in a bin: its center, radius, exposed height, weight and pixel window
// [c0, c1) x [r0, r1). 64 bytes, so bins copy to shared memory in 16-byte units.
struct BoulderEntry {
    double x, y, radius, exposed, weight;
    int32_t c0, c1, r0, r1;
    double pad_;
};
static_assert(sizeof(BoulderEntry) == 64, "BoulderEntry must be a multiple of 16 bytes");

struct BoulderBins {
    uint32_t binsX, binsY;
    uint32_t* counts;  // [bins + 1]
    uint32_t* cursor;  // [bins]
    BoulderEntry* entries;
    uint32_t capacity;
    int4* windows;     // [boulders]
    uint32_t firstBin; // the bin of a launch's first block (a strip of bin rows)
};

cudaError_t launch_boulder_count(const BoulderRecord* boulders, uint32_t n, const Grid& grid,
                                 double width, const BoulderBins& bins, cudaStream_t stream);
cudaError_t launch_boulder_scatter(const BoulderRecord* boulders, uint32_t n,
                                   const BoulderBins& bins, cudaStream_t stream);
cudaError_t launch_boulder_bake(const Grid& grid, double width, NoData nodata,
                                const BoulderBins& bins, float* heights, uint32_t* flags,
                                cudaStream_t stream, uint32_t firstBinRow = 0,
                                uint32_t binRows = 0xffffffffu, uint32_t polls = kWaitPolls);

// --- diamond-square ----------------------------------------------------------------------
// Where the finest nodes lie: node (0, 0) and the node steps along x and y (north up).
struct DsFrame {
    double originX, originY, stepX, stepY;
};
constexpr int kMaxDsLevels = 30;
#ifndef TGB_DS_THREADS
#define TGB_DS_THREADS 256
#endif
constexpr uint32_t kDsTileThreads = TGB_DS_THREADS;  // threads of a diamond-square CTA
// One refinement job: `levels` refinements of the posts read at every cell of `grid` into
// `heights` (row-major, `pitch` floats a row), a CTA per blockW x blockH cells (sides at most 64);
// or, with `points` set, at each of `blocks` points (x, y pairs), a CTA per point, point k's
// height at heights[pointIndex[k]] (heights[k] without an index). launch_ds_tiles runs one job
// with posts from an array; the batch engine runs many with posts from its source.
struct DsTile {
    Grid grid;
    DsFrame frame;                           // the finest level's
    int levels;
    uint32_t seed;
    uint32_t blockW, blockH, blocksX, pitch;
    uint32_t blocks;                         // blocks of the job
    uint32_t capEven, capOdd;                // doubles of the even / odd levels' shared buffers
    double squareStep[kMaxDsLevels + 1];     // displacement scale per level (index 1..levels)
    double diamondStep[kMaxDsLevels + 1];
    const float* posts;                      // the lattice's columns col0.. and rows row0..
    int64_t col0, row0;
    uint32_t pw, ph;
    double postSpacing;                      // posts from a source: node (c, r) at (c, r) * this
    const double* points;                    // point jobs: the points
    const uint32_t* pointIndex;              // point jobs: where each one's height goes
    uint64_t heightOffset;                   // batch jobs: heights of the batch's output
    float* heights;
    uint32_t* status;                        // flag 1: a block's boxes outgrew their buffers
};
// Shared bytes of a diamond-square CTA's node buffers: three CTAs share an SM.
#ifndef TGB_DS_SHARED_BUDGET
#define TGB_DS_SHARED_BUDGET (72 * 1024)
#endif
constexpr size_t kDsSharedBudget = TGB_DS_SHARED_BUDGET;
// The refinement of posts on `postGrid` (a lattice: post (0, 0) at its cell (0, 0)) read at
// `grid`'s cells (Levels, the frame and Displacement, diamond_square.cpp:289-389): fills t's
// grid, frame, levels, seed, displacement scales, pitch (grid.width), block shape and blocks;
// with `single`, the buffers of a one-cell block (a point). False when no block's node buffers
// fit kDsSharedBudget.
bool ds_setup(DsTile& t, const Grid& postGrid, double fractalDimension, double scale,
              uint32_t seed, double minPixelSize, bool spline, const Grid& grid,
              bool single = false);
cudaError_t launch_ds_tiles(const DsTile& t, bool spline, cudaStream_t stream);
// Philox4x32-10 of n (counter, key) sextets, and the displacement normal the first two counter
// words, the third's low 5 bits and the key's first word key as (col, row, level, seed).
cudaError_t launch_philox_probe(const uint32_t* in, uint32_t n, uint32_t* out, double* normals,
                                cudaStream_t stream);

// --- batched tiles and point sets (batch.cu) ----------------------------------------------
// Many tiles and point sets evaluated together: source fBm, craters and boulders of every item in
// one persistent launch over all the items' bins, after one count / scan / scatter per feature
// kind.

constexpr int kBatchMaxOctaves = 32;

// One tile (a grid) or one point set of a batch. Its bins are numbered binBase .. binBase +
// binsX * binsY - 1 in the batch's bin order, which is the work queue's order. A point set's
// "bins" are blocks of consecutive points (binsY = 1), its points at points[pointBase ..] and its
// heights at heightOffset + i; grid.width holds its point count.
struct BatchTile {
    Grid grid;
    uint64_t heightOffset;  // output index of cell (0, 0) or of point 0
    uint32_t pitch;         // output floats from one row to the next
    uint32_t binsX, binsY;
    uint32_t binBase;
    uint32_t anchorBase;    // the tile's first OctaveAnchor
    uint32_t pointBase;     // point sets: first point; ~0u for a grid
    double boulderWidth;    // dome band width (the tile's sample spacing)
    uint32_t kind;          // kTileGrid, kTilePoints or kTileIndexedPoints
    uint32_t tableBase;     // indexed points: their region table (see below)
};
static_assert(sizeof(BatchTile) == 104, "BatchTile layout");

// Item kinds: a grid; a point set whose blocks are binned like a grid's bins; a point set whose
// craters come from resident per-region cell lists (PointRegion), one point per thread. An
// indexed point set's regions cover its bounding box: region (ix, iy) is pointTable[tableBase +
// (iy - iy0) * tableWidth + (ix - ix0)] (a PointRegion index, ~0u for none), with ix0 * side and
// iy0 * side in grid.originX / grid.originY, the region side in grid.pixelWidth, tableWidth in
// grid.height and the table's rows in pitch; its points keep the caller's order.
constexpr uint32_t kTileGrid = 0, kTilePoints = 1, kTileIndexedPoints = 2;

// A resident feature region as indexed points read it: its square of g x g cells of side `cell`
// from (x0, y0), each cell listing the records (relative to recBase) whose footprint disk meets
// it: lists[listBase + c] .. lists[listBase + c + 1] index lists[listBase + g * g + 1 + k].
struct PointRegion {
    double x0, y0, cell;
    uint32_t recBase, dataBase, listBase, g;
};
static_assert(sizeof(PointRegion) == 40, "PointRegion layout");

// A run of crater records and boulders one tile (or point set) takes: records [recordBegin,
// recordBegin + recordCount) with data offsets relative to data + dataBase, boulders [boulderBegin,
// boulderBegin + boulderCount). Several refs may name the same records (regions shared by tiles).
// recordPairs / boulderPairs are the refs' exclusive prefix sums of the counts: the batch's
// (ref, record) pairs are numbered by them.
struct BatchRef {
    uint32_t tile;
    uint32_t recordBegin, recordCount, dataBase;
    uint32_t boulderBegin, boulderCount;
    uint32_t recordPairs, boulderPairs;
};
static_assert(sizeof(BatchRef) == 32, "BatchRef layout");

// The lattice position of a tile's cell (0, 0) for one octave, split in double into an integer
// cell (ix, iy) and a float fraction (fx, fy), and the lattice steps of one column (ax, bx) and
// one row (ay, by): cell (c, r) lies at (ix + fx + c ax + r ay, iy + fy + c bx + r by).
struct OctaveAnchor {
    int32_t ix, iy;
    float fx, fy;
    float ax, ay, bx, by;
};
static_assert(sizeof(OctaveAnchor) == 32, "OctaveAnchor layout");

// The batch's source: elevation + amplitude * (sum of weight * Perlin octave) / total. Points take
// each octave's lattice position in double from the rotation (tc, ts), frequency and offsets.
struct BatchNoise {
    int32_t octaves;
    float amplitude, total, elevation;
    uint32_t baseInOutput;  // 1: the source is already in the output (a diamond-square pass)
    double scale;  // amplitude / total
    uint32_t seedTerm[kBatchMaxOctaves];  // octave seed through pcg3d's first LCG step
    float weight[kBatchMaxOctaves];
    double tc[kBatchMaxOctaves], ts[kBatchMaxOctaves], frequency[kBatchMaxOctaves];
    double ox[kBatchMaxOctaves], oy[kBatchMaxOctaves];
};

// Per-run values the launches read from device memory, so one captured graph serves any batch
// within the plan's capacities.
struct BatchHeader {
    uint32_t tiles, refs, bins, pad_;
    uint32_t refRecords, refBoulders;    // (ref, record) and (ref, boulder) pairs in all
    float* heights;
    uint32_t next;     // work-queue cursor
    uint32_t flags;    // 1 datum seen, 2 staged copy timed out, 8 a record needs the general path
    unsigned long long craterPairs, boulderPairs;  // (cell, feature) pairs evaluated
    uint32_t craterEntries, boulderEntries;         // entries the bins needed
    uint32_t dsJobs, dsBlocks;                      // the diamond-square pass: grid jobs, blocks
    uint32_t dsPointJobs, dsPoints;                 // and point-set jobs, points
    uint32_t evalEnd, pad2_;                        // the evaluation takes bins below this
};

struct BatchView {
    BatchHeader* header;
    const BatchTile* tiles;
    const BatchRef* refs;
    const OctaveAnchor* anchors;
    const double* points;          // (x, y) per point of every point set, blocks spatially sorted
    const uint32_t* pointIndex;    // the caller's index of each point within its set
    const double* pointBoxes;      // (min x, min y, max x, max y) per point-set bin
    const CraterRecord* records;
    const double* footprints;      // optional (x, y, reach) per record
    const float* data;
    float* harmonics;              // mirrors data
    const BoulderRecord* boulders;
    uint32_t* craterCounts;        // [capacityBins + 1]
    uint32_t* craterCursor;        // [capacityBins]
    BinEntry* craterEntries;
    uint32_t craterCapacity;
    int4* craterBoxes;             // [record pairs]
    float* craterCulls;            // [record pairs]
    uint32_t* boulderCounts;
    uint32_t* boulderCursor;
    BoulderEntry* boulderEntries;
    uint32_t boulderCapacity;
    int4* boulderWindows;          // [boulder pairs]
    uint32_t capacityBins;
    uint32_t harmonicsReady;       // the harmonics are already in place (resident regions)
    const uint32_t* pointTable;    // indexed points: region tables
    const PointRegion* pointRegions;
    const uint32_t* pointLists;    // the regions' cell lists
    const float* culls;            // indexed points: each record's cull distance
    const DsTile* dsJobs;          // diamond-square source: one job per grid item
    const uint32_t* dsFirst;       // [jobs + 1]: each job's first block of the pass
    const DsTile* dsPointJobs;     // one job per point set
    const uint32_t* dsPointFirst;  // [point jobs + 1]: each job's first point of the pass
};

// A kernel shape of the persistent evaluation: bins of binW x binH cells (point sets: blocks of
// binW x binH points), cellsPerThread adjacent cells of one row per thread.
struct BatchVariant {
    uint32_t binW, binH, cellsPerThread;
};
// The variants compiled in; variant 0 also serves batches that need the general shaping path.
int batch_variant_count();
BatchVariant batch_variant(int index);
// Persistent CTAs of `index` that fit on one SM (occupancy), for sizing the launch.
int batch_blocks_per_sm(int index, bool fast);

// Counting and scattering of the batch's (ref, record) and (ref, boulder) pairs into its bins,
// for `variant`'s bin size (launches sized for `maxRecordPairs` / `maxBoulderPairs`, counts read
// from the header).
cudaError_t launch_batch_bin(const CraterShapeKernel& k, const BatchView& v,
                             const BatchVariant& variant, uint32_t maxRecordPairs,
                             uint32_t maxBoulderPairs, uint32_t* scanScratch, cudaStream_t stream);
// The diamond-square source of a batch (header->dsJobs grid jobs over header->dsBlocks blocks,
// header->dsPointJobs point-set jobs over header->dsPoints points): persistent CTAs take the
// grid blocks in turn and, in a second launch, their warps take the points one each, each job's
// level-0 nodes from the batch's fBm at its post lattice, and write every item's base heights
// into the output before the evaluation adds the layers (noise.baseInOutput). A block whose node
// boxes outgrow the shared buffers sets header flag 16 and writes nothing.
// A point's node pyramid in doubles, both buffers (one warp's share of the points' launch).
constexpr uint32_t kDsPointPool = 768;
// batch_ds_setup lets the pass take its shared memory and gives the CTAs of a launch (call it
// before any capture).
cudaError_t batch_ds_setup(uint32_t& ctas);
cudaError_t launch_batch_ds(const BatchNoise& noise, const BatchView& v, bool spline,
                            uint32_t ctas, cudaStream_t stream);
// The persistent evaluation over every bin of the batch, `ctas` CTAs.
cudaError_t launch_batch_evaluate(const CraterShapeKernel& k, const BatchNoise& noise,
                                  const BatchView& v, int variant, bool fast, uint32_t ctas,
                                  cudaStream_t stream);

// The ALU issue-rate probe (probe.cu): one launch of a fixed IMAD/FFMA mix; `laneOps` receives
// the lane operations it performs.
cudaError_t launch_alu_probe(uint32_t* sink, uint64_t* laneOps, cudaStream_t stream);

// Exclusive prefix sum of n counts in place, writing the total to counts[n]. `scratch` holds
// scan_scratch_words(n) words.
size_t scan_scratch_words(uint32_t n);
cudaError_t launch_exclusive_scan(uint32_t* counts, uint32_t n, uint32_t* scratch,
                                  cudaStream_t stream);

}  // namespace tgb
