// The batched form's host engine, shared by the C ABI (batch_api.cu) and the request server
// (serve.cu): a batch is a list of items (tiles and point sets), refs naming runs of crater
// records and boulders in device arrays, and the source; the engine numbers the bins, sizes its
// buffers, captures the binning and the persistent evaluation as CUDA graphs and replays them.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/tgb200.h"
#include "kernels.h"

namespace tgb {
namespace batch {

// Per-octave lattice constants in double (the FP64 form of Fractal2's recurrences) for the
// anchors of grid items.
struct Octave {
    double frequency, tc, ts, ox, oy;
};

// The source of a batch from `n` Fractals (at most one enabled: a Perlin fBm without warp).
int make_noise(const void* fractals, uint32_t n, float elevation, BatchNoise& noise,
               std::vector<Octave>& octaves);

// An item before bin numbering: a grid tile, or a point set (points = true) whose points are
// [pointBegin, pointBegin + grid.width) of the batch's device-order points.
struct Item {
    Grid grid;
    uint64_t heightOffset;
    uint32_t pitch;
    bool points;
    uint32_t pointBegin;
    double boulderWidth;
    uint32_t kind = kTileGrid;  // kTileGrid, kTilePoints or kTileIndexedPoints
    uint32_t tableBase = 0;     // indexed points: their region table in Spec::pointTable
    double dsSpacing = 0.0;     // point sets under a diamond-square source: the spacing read at
};

// A diamond-square source in place of the fBm at every cell (DiamondSquareUpsampler over a DEM,
// src/sources/diamond_square.cpp:488-516): the batch's fBm sampled at a post lattice of
// `postSpacing` (post (i, j) at (i, -j) * postSpacing, node (i, j) of level 0 at (i, j) *
// postSpacing), rounded to float as a DEM's posts, refined to each item's spacing (point sets:
// Item::dsSpacing) with DiamondSquareOptions' fractal dimension, scale, seed, minimum pixel size
// and interpolation.
struct DsSource {
    bool on = false;
    double postSpacing = 0.0;
    double fractalDimension = 2.2, scale = 0.0, minPixelSize = 0.0;
    uint32_t seed = 0;
    bool spline = false;
};

// Device arrays the refs index; the batch reads them and owns none.
struct Features {
    const CraterRecord* records = nullptr;
    const double* footprints = nullptr;
    const float* data = nullptr;
    float* harmonics = nullptr;  // as long as data
    const BoulderRecord* boulders = nullptr;
    bool harmonicsReady = false;  // harmonics already computed (no per-batch pass)
    const uint32_t* pointLists = nullptr;  // indexed points: resident cell lists
    const float* culls = nullptr;          // indexed points: cull distance per record
};

// A whole batch, host side. `points` holds (x, y) per point in device order (each set's points
// spatially sorted) and `pointIndex` each one's index in its caller's set.
struct Spec {
    std::vector<Item> items;
    std::vector<BatchRef> refs;  // recordPairs / boulderPairs filled by the engine
    std::vector<double> points;
    std::vector<uint32_t> pointIndex;
    std::vector<PointRegion> pointRegions;  // indexed points: the regions they read
    std::vector<uint32_t> pointTable;       // indexed points: region tables (kernels.h)
    BatchNoise noise{};
    std::vector<Octave> octaves;
    DsSource ds;
    CraterShapeKernel kernel{};
    bool fast = true;
    Features features;
};

// Sorts one point set's points along a Morton curve: appends them to spec.points and their
// caller indices to spec.pointIndex.
void append_points(Spec& spec, const double* xy, uint32_t count);

// Loads `spec` (its feature arrays already on the device) into the batch: uploads items, refs,
// anchors and points, numbers the bins. The spec is moved in.
int load(tg_batch* b, Spec&& spec);

// Enqueues one evaluation of the loaded batch into `out` on `stream` (binning graph, then
// evaluation graph); `finish` waits for it, checks its status and, when the bins needed more
// entries than they held, grows them and evaluates again.
int launch(tg_batch* b, float* out, cudaStream_t stream);
int finish(tg_batch* b);
// Whether the last launch has finished (without waiting).
bool done(tg_batch* b);

size_t output_floats(const tg_batch* b);
uint64_t cells(const tg_batch* b);
// Graph launches so far (a finish that re-launched for more entries adds one).
uint32_t replays(const tg_batch* b);
// Device bytes the batch's buffers hold.
size_t device_bytes(const tg_batch* b);

}  // namespace batch
}  // namespace tgb
