// The batched form's C ABI (tg_batch_* in include/tgb200.h) and engine (batch_internal.h):
// input checks, the source's octave constants and per-tile lattice anchors (double), point sets
// in Morton order, the bin numbering and queue order, device buffers sized by capacity, CUDA
// graph capture and replay, and the autotuner over kernel shapes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "batch_internal.h"
#include "kernels.h"

using namespace tgb;
using namespace tgb::api;
using namespace tgb::batch;

namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kLcgA = 1664525u, kLcgC = 1013904223u;
// The octave lattice turn (include/terraingen/noise/fractal.h:146-148) as floats.
constexpr float kTurnCos = -0.7373688780783197f;
constexpr float kTurnSin = 0.6754902942615238f;

void pcg3d(uint32_t v[3]) {  // include/terraingen/noise/hash.h:40
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
}

enum BatchSlot {
    kSlotTiles,
    kSlotRefs,
    kSlotAnchors,
    kSlotPoints,
    kSlotPointIndex,
    kSlotPointBoxes,
    kSlotPointTable,
    kSlotPointRegions,
    kSlotRecords,
    kSlotFootprints,
    kSlotData,
    kSlotHarmonics,
    kSlotBoulders,
    kSlotCraterCounts,
    kSlotCraterCursor,
    kSlotCraterEntries,
    kSlotCraterBoxes,
    kSlotCraterCulls,
    kSlotBoulderCounts,
    kSlotBoulderCursor,
    kSlotBoulderEntries,
    kSlotBoulderWindows,
    kSlotScanScratch,
    kSlotHeader,
    kSlotOutput,
    kSlotDsJobs,
    kSlotDsFirst,
    kSlotDsPointJobs,
    kSlotDsPointFirst,
    kBatchSlotCount
};

// Chunks of a batch whose heights go to host memory: each one's copy overlaps the next one's
// evaluation.
constexpr int kOutputChunks = 8;

// What a captured graph depends on; a change means a new capture.
struct Signature {
    BatchView view;
    int variant;
    bool fast;
    uint32_t ctas, maxRecordPairs, maxBoulderPairs;
    CraterShapeKernel kernel;
    BatchNoise noise;
    uint32_t dsCtas, dsSpline;  // the diamond-square pass's CTAs (0: none), Catmull-Rom (1)
};

}  // namespace

struct tg_batch {
    tg_device* dev = nullptr;
    cudaStream_t stream = nullptr;
    // Recorded before the binning graph, between it and the evaluation graph, and after.
    cudaEvent_t events[3] = {nullptr, nullptr, nullptr};
    BatchHeader* pinned = nullptr;  // [0] written before each launch, [1] read back after
    Buffer slots[kBatchSlotCount];
    int variant = 0;

    bool loaded = false;
    Spec spec;
    std::vector<BatchTile> tiles;   // spec.items numbered for the current variant
    uint32_t dsJobs = 0, dsBlocks = 0, dsCtas = 0;  // the diamond-square pass: grid jobs
    uint32_t dsPointJobs = 0, dsPoints = 0;          // and point-set jobs
    uint32_t bins = 0;
    uint32_t recordPairs = 0, boulderPairs = 0;
    size_t outputFloats = 0;
    uint64_t cells = 0;

    // The launch in flight.
    bool pending = false;
    float* out = nullptr;
    cudaStream_t launchStream = nullptr;
    Signature launched{};

    cudaGraph_t graph[2] = {nullptr, nullptr};  // binning, evaluation

    // Host outputs: the evaluation by chunks of items, each chunk's heights copied out on
    // `copyStream` while the next chunk is evaluated (made on the first such call).
    cudaStream_t copyStream = nullptr;
    cudaEvent_t chunkDone[kOutputChunks] = {};
    uint32_t* chunkWords = nullptr;  // pinned: each chunk's first bin and end bin
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    Signature captured{};
    uint32_t captures = 0, replays = 0;
    tg_batch_stats last{};
};

namespace {

template <typename T>
T* ptr(tg_batch* b, BatchSlot s) {
    return static_cast<T*>(b->slots[s].ptr);
}

template <typename T>
uint32_t capacity(tg_batch* b, BatchSlot s) {
    const size_t n = b->slots[s].bytes / sizeof(T);
    return uint32_t(std::min<size_t>(n, 0xffffffffu));
}

int effective_variant(const tg_batch* b) {
    return b->spec.fast ? b->variant : 0;
}

template <typename T>
int upload(tg_batch* b, BatchSlot slot, const T* src, size_t count) {
    if (count == 0) {
        return TG_OK;
    }
    TG_CUDA(b->slots[slot].reserve(count * sizeof(T)), "allocation");
    TG_CUDA(cudaMemcpyAsync(b->slots[slot].ptr, src, count * sizeof(T), cudaMemcpyHostToDevice,
                            b->stream),
            "copy to device");
    return TG_OK;
}

uint32_t capacity_bins(tg_batch* b) {
    return std::min({capacity<uint32_t>(b, kSlotCraterCounts),
                     capacity<uint32_t>(b, kSlotCraterCursor),
                     capacity<uint32_t>(b, kSlotBoulderCounts),
                     capacity<uint32_t>(b, kSlotBoulderCursor)}) - 1;
}

// Numbers the loaded items' bins for the current kernel shape, bounds each point block, and
// uploads the tile table and the blocks' boxes.
int plan_bins(tg_batch* b) {
    const BatchVariant v = batch_variant(effective_variant(b));
    const uint32_t block = v.binW * v.binH;  // points per point-set block
    const Spec& spec = b->spec;
    std::vector<BatchTile> out(spec.items.size());
    std::vector<double> boxes;
    uint64_t base = 0;
    const int stride = std::max(spec.noise.octaves, 1);
    for (size_t i = 0; i < spec.items.size(); ++i) {
        const Item& it = spec.items[i];
        BatchTile& d = out[i];
        d.grid = it.grid;
        d.heightOffset = it.heightOffset;
        d.pitch = it.pitch;
        d.binBase = uint32_t(base);
        d.anchorBase = uint32_t(i) * uint32_t(stride);
        d.boulderWidth = it.boulderWidth;
        d.kind = it.kind;
        d.tableBase = it.tableBase;
        if (it.kind == kTileIndexedPoints) {
            // One point per thread of the kernel shape.
            const uint32_t threads = v.binW * v.binH / v.cellsPerThread;
            d.pointBase = it.pointBegin;
            d.binsX = (it.grid.width + threads - 1) / threads;
            d.binsY = 1;
        } else if (it.points) {
            d.pointBase = it.pointBegin;
            d.binsX = (it.grid.width + block - 1) / block;
            d.binsY = 1;
            // Boxes are indexed by bin: pad up to this item's first bin.
            boxes.resize(size_t(base) * 4, 0.0);
            for (uint32_t q = 0; q < d.binsX; ++q) {
                double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
                const uint32_t end = std::min(it.grid.width, (q + 1) * block);
                for (uint32_t p = q * block; p < end; ++p) {
                    const double* xy = &spec.points[2 * (size_t(it.pointBegin) + p)];
                    lo[0] = std::min(lo[0], xy[0]);
                    lo[1] = std::min(lo[1], xy[1]);
                    hi[0] = std::max(hi[0], xy[0]);
                    hi[1] = std::max(hi[1], xy[1]);
                }
                boxes.insert(boxes.end(), {lo[0], lo[1], hi[0], hi[1]});
            }
        } else {
            d.pointBase = kNone;
            d.binsX = (it.grid.width + v.binW - 1) / v.binW;
            d.binsY = (it.grid.height + v.binH - 1) / v.binH;
        }
        base += uint64_t(d.binsX) * d.binsY;
    }
    if (base >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "a batch holds fewer than 2^32 bins");
    }
    b->bins = uint32_t(base);
    b->tiles = out;
    const size_t words = size_t(b->bins) + 1;
    TG_CUDA(b->slots[kSlotCraterCounts].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotCraterCursor].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotBoulderCounts].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotBoulderCursor].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotScanScratch].reserve(scan_scratch_words(capacity_bins(b)) *
                                               sizeof(uint32_t)),
            "allocation");
    if (int s = upload(b, kSlotTiles, out.data(), out.size())) {
        return s;
    }
    if (!boxes.empty()) {
        boxes.resize(size_t(b->bins) * 4, 0.0);
        if (int s = upload(b, kSlotPointBoxes, boxes.data(), boxes.size())) {
            return s;
        }
    }
    TG_CUDA(cudaStreamSynchronize(b->stream), "synchronize");
    return TG_OK;
}

BatchView make_view(tg_batch* b) {
    const Features& f = b->spec.features;
    BatchView v{};
    v.header = ptr<BatchHeader>(b, kSlotHeader);
    v.tiles = ptr<BatchTile>(b, kSlotTiles);
    v.refs = ptr<BatchRef>(b, kSlotRefs);
    v.anchors = ptr<OctaveAnchor>(b, kSlotAnchors);
    v.points = ptr<double>(b, kSlotPoints);
    v.pointIndex = ptr<uint32_t>(b, kSlotPointIndex);
    v.pointBoxes = ptr<double>(b, kSlotPointBoxes);
    v.records = f.records;
    v.footprints = f.footprints;
    v.data = f.data;
    v.harmonics = f.harmonics;
    v.boulders = f.boulders;
    v.craterCounts = ptr<uint32_t>(b, kSlotCraterCounts);
    v.craterCursor = ptr<uint32_t>(b, kSlotCraterCursor);
    v.craterEntries = ptr<BinEntry>(b, kSlotCraterEntries);
    v.craterCapacity = capacity<BinEntry>(b, kSlotCraterEntries);
    v.craterBoxes = ptr<int4>(b, kSlotCraterBoxes);
    v.craterCulls = ptr<float>(b, kSlotCraterCulls);
    v.boulderCounts = ptr<uint32_t>(b, kSlotBoulderCounts);
    v.boulderCursor = ptr<uint32_t>(b, kSlotBoulderCursor);
    v.boulderEntries = ptr<BoulderEntry>(b, kSlotBoulderEntries);
    v.boulderCapacity = capacity<BoulderEntry>(b, kSlotBoulderEntries);
    v.boulderWindows = ptr<int4>(b, kSlotBoulderWindows);
    v.capacityBins = capacity_bins(b);
    v.harmonicsReady = f.harmonicsReady ? 1u : 0u;
    v.pointTable = ptr<uint32_t>(b, kSlotPointTable);
    v.pointRegions = ptr<PointRegion>(b, kSlotPointRegions);
    v.pointLists = f.pointLists;
    v.culls = f.culls;
    v.dsJobs = ptr<DsTile>(b, kSlotDsJobs);
    v.dsFirst = ptr<uint32_t>(b, kSlotDsFirst);
    v.dsPointJobs = ptr<DsTile>(b, kSlotDsPointJobs);
    v.dsPointFirst = ptr<uint32_t>(b, kSlotDsPointFirst);
    return v;
}

Signature signature(tg_batch* b) {
    Signature s;
    std::memset(&s, 0, sizeof(s));
    const BatchView view = make_view(b);
    std::memcpy(&s.view, &view, sizeof(view));
    s.variant = effective_variant(b);
    s.fast = b->spec.fast;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev->ordinal);
    s.ctas = uint32_t(sms * batch_blocks_per_sm(s.variant, s.fast));
    s.maxRecordPairs =
        std::min(capacity<int4>(b, kSlotCraterBoxes), capacity<float>(b, kSlotCraterCulls));
    s.maxBoulderPairs = capacity<int4>(b, kSlotBoulderWindows);
    std::memcpy(&s.kernel, &b->spec.kernel, sizeof(s.kernel));
    std::memcpy(&s.noise, &b->spec.noise, sizeof(s.noise));
    s.dsCtas = b->spec.ds.on ? b->dsCtas : 0u;
    s.dsSpline = b->spec.ds.on && b->spec.ds.spline ? 1u : 0u;
    return s;
}

void drop_graph(tg_batch* b) {
    for (int i = 0; i < 2; ++i) {
        if (b->exec[i] != nullptr) {
            cudaGraphExecDestroy(b->exec[i]);
            b->exec[i] = nullptr;
        }
        if (b->graph[i] != nullptr) {
            cudaGraphDestroy(b->graph[i]);
            b->graph[i] = nullptr;
        }
    }
}

// Ends a capture begun on the batch's stream and instantiates it as graph `i`.
int finish_capture(tg_batch* b, int i, cudaError_t err) {
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(b->stream, &graph);
    if (err != cudaSuccess) {
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        return cuda_fail(err, "batch capture");
    }
    TG_CUDA(end, "end capture");
    b->graph[i] = graph;
    TG_CUDA(cudaGraphInstantiate(&b->exec[i], graph, 0), "graph instantiate");
    return TG_OK;
}

// Captures two graphs: the header upload and the binning (count, scan, scatter), then the
// persistent evaluation and the status read-back. Launched back to back; events between them
// time each part.
int capture(tg_batch* b, const Signature& s) {
    drop_graph(b);
    (void)cudaGetLastError();  // a stale launch error must not be read as one of this capture's
    TG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaMemcpyAsync(s.view.header, &b->pinned[0], sizeof(BatchHeader),
                                      cudaMemcpyHostToDevice, b->stream);
    if (err == cudaSuccess) {
        err = launch_batch_bin(s.kernel, s.view, batch_variant(s.variant), s.maxRecordPairs,
                               s.maxBoulderPairs, ptr<uint32_t>(b, kSlotScanScratch), b->stream);
    }
    if (int st = finish_capture(b, 0, err)) {
        return st;
    }
    TG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    err = s.dsCtas != 0u ? launch_batch_ds(s.noise, s.view, s.dsSpline != 0u, s.dsCtas, b->stream)
                         : cudaSuccess;
    if (err == cudaSuccess) {
        err = launch_batch_evaluate(s.kernel, s.noise, s.view, s.variant, s.fast, s.ctas,
                                    b->stream);
    }
    if (err == cudaSuccess) {
        err = cudaMemcpyAsync(&b->pinned[1], s.view.header, sizeof(BatchHeader),
                              cudaMemcpyDeviceToHost, b->stream);
    }
    if (int st = finish_capture(b, 1, err)) {
        return st;
    }
    b->captured = s;
    ++b->captures;
    return TG_OK;
}

int check_batch(tg_batch* b) {
    if (b == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "batch is null");
    }
    return check_device(b->dev);
}

// The (x, y) of a point set scaled to 16-bit cells of its bounding box, bits interleaved.
uint32_t morton(double x, double y, const double* lo, const double* scale) {
    auto spread = [](uint32_t v) {
        v &= 0xffffu;
        v = (v | (v << 8)) & 0x00ff00ffu;
        v = (v | (v << 4)) & 0x0f0f0f0fu;
        v = (v | (v << 2)) & 0x33333333u;
        v = (v | (v << 1)) & 0x55555555u;
        return v;
    };
    const uint32_t qx = uint32_t(std::min(65535.0, std::max(0.0, (x - lo[0]) * scale[0])));
    const uint32_t qy = uint32_t(std::min(65535.0, std::max(0.0, (y - lo[1]) * scale[1])));
    return spread(qx) | (spread(qy) << 1);
}

}  // namespace

namespace tgb {
namespace batch {

int make_noise(const void* fractals, uint32_t n, float elevation, BatchNoise& noise,
               std::vector<Octave>& octaves) {
    noise = BatchNoise{};
    octaves.clear();
    noise.elevation = elevation;
    noise.total = 1.0f;
    noise.scale = 0.0;
    const Fractal* only = nullptr;
    for (uint32_t i = 0; i < n; ++i) {
        const Fractal* f = static_cast<const Fractal*>(fractals) + i;
        if (!f->enabled) {
            continue;
        }
        if (only != nullptr) {
            return fail(TG_ERROR_UNSUPPORTED, "a batch's source is one fractal");
        }
        only = f;
    }
    if (only == nullptr) {
        return TG_OK;
    }
    if (only->basis != kBasisPerlin || only->type != kTypeFbm || only->warpAmplitude > 0.0f) {
        return fail(TG_ERROR_UNSUPPORTED, "a batch's source is a Perlin fBm without warp");
    }
    if (only->octaves < 1 || only->octaves > kBatchMaxOctaves || !(only->wavelength > 0.0f) ||
        !(only->lacunarity > 1.0f) || !(only->gain > 0.0f)) {
        return fail(TG_ERROR_ARGUMENT, "the fractal is invalid");
    }
    // Fractal2's octaves (fractal.h:219-240): weights in float as the reference accumulates
    // them; frequency, turn and offsets in double for the lattice positions.
    noise.octaves = only->octaves;
    noise.amplitude = only->amplitude;
    float weight = 1.0f, total = 0.0f;
    double frequency = 1.0 / double(only->wavelength);
    double tc = 1.0, ts = 0.0;
    for (int o = 0; o < only->octaves; ++o) {
        uint32_t h[3] = {only->seed, uint32_t(o), 0u};
        pcg3d(h);
        noise.seedTerm[o] = h[0] * kLcgA + kLcgC;
        noise.weight[o] = weight;
        total += weight;
        weight *= only->gain;
        Octave oc;
        oc.frequency = frequency;
        oc.tc = tc;
        oc.ts = ts;
        oc.ox = double(float(h[1] >> 8u) * 0x1p-24f);
        oc.oy = double(float(h[2] >> 8u) * 0x1p-24f);
        octaves.push_back(oc);
        noise.tc[o] = tc;
        noise.ts[o] = ts;
        noise.frequency[o] = frequency;
        noise.ox[o] = oc.ox;
        noise.oy[o] = oc.oy;
        frequency *= double(only->lacunarity);
        const double c = double(kTurnCos), s = double(kTurnSin);
        const double nc = tc * c - ts * s;
        ts = ts * c + tc * s;
        tc = nc;
    }
    noise.total = total;
    noise.scale = double(noise.amplitude) / double(total);
    return TG_OK;
}

void append_points(Spec& spec, const double* xy, uint32_t count) {
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (uint32_t i = 0; i < count; ++i) {
        lo[0] = std::min(lo[0], xy[2 * i]);
        lo[1] = std::min(lo[1], xy[2 * i + 1]);
        hi[0] = std::max(hi[0], xy[2 * i]);
        hi[1] = std::max(hi[1], xy[2 * i + 1]);
    }
    const double scale[2] = {hi[0] > lo[0] ? 65535.0 / (hi[0] - lo[0]) : 0.0,
                             hi[1] > lo[1] ? 65535.0 / (hi[1] - lo[1]) : 0.0};
    // (Morton code, index) in one word: sorting the words orders by code, ties by index.
    std::vector<uint64_t> key(count);
    for (uint32_t i = 0; i < count; ++i) {
        key[i] = (uint64_t(morton(xy[2 * i], xy[2 * i + 1], lo, scale)) << 32) | i;
    }
    std::sort(key.begin(), key.end());
    const size_t at = spec.pointIndex.size();
    spec.points.resize(2 * (at + count));
    spec.pointIndex.resize(at + count);
    for (uint32_t n = 0; n < count; ++n) {
        const uint32_t i = uint32_t(key[n]);
        spec.points[2 * (at + n)] = xy[2 * i];
        spec.points[2 * (at + n) + 1] = xy[2 * i + 1];
        spec.pointIndex[at + n] = i;
    }
}

// The diamond-square pass's jobs, one per item (after the points are on the device): a grid
// item's blocks, or a point set's points, each written at its item's output offset.
int load_ds(tg_batch* b) {
    Spec& s = b->spec;
    s.noise.baseInOutput = s.ds.on ? 1u : 0u;
    b->dsJobs = 0;
    b->dsBlocks = 0;
    b->dsPointJobs = 0;
    b->dsPoints = 0;
    if (!s.ds.on) {
        return TG_OK;
    }
    const double P = s.ds.postSpacing;
    if (!(P > 0.0) || !std::isfinite(P) || !(s.ds.fractalDimension >= 2.0) ||
        !(s.ds.fractalDimension <= 3.0) || !(s.ds.scale >= 0.0) || !(s.ds.minPixelSize >= 0.0)) {
        return fail(TG_ERROR_ARGUMENT, "diamond-square source: post spacing > 0, fractal "
                                       "dimension in [2, 3], scale and min pixel size >= 0");
    }
    TG_CUDA(batch_ds_setup(b->dsCtas), "diamond-square set-up");
    // The post lattice as a grid whose cell (0, 0) is centered on the origin.
    const Grid lattice{1u, 1u, -0.5 * P, P, 0.0, 0.5 * P, 0.0, -P};
    uint32_t* flags = &ptr<BatchHeader>(b, kSlotHeader)->flags;
    std::vector<DsTile> jobs, pointJobs;
    std::vector<uint32_t> first, pointFirst;
    jobs.reserve(s.items.size());
    uint64_t blocks = 0, points = 0;
    for (const Item& it : s.items) {
        DsTile t{};
        if (it.points) {
            const double d = it.dsSpacing;
            if (!(d > 0.0) || !std::isfinite(d)) {
                return fail(TG_ERROR_ARGUMENT, "point sets under a diamond-square source need "
                                               "the spacing they are read at");
            }
            const Grid one{1u, 1u, -0.5 * d, d, 0.0, 0.5 * d, 0.0, -d};
            if (!ds_setup(t, lattice, s.ds.fractalDimension, s.ds.scale, s.ds.seed,
                          s.ds.minPixelSize, s.ds.spline, one, true) ||
                t.capEven + t.capOdd > kDsPointPool) {
                return fail(TG_ERROR_ARGUMENT, "the points are too coarse for the posts' nodes");
            }
            t.points = ptr<double>(b, kSlotPoints) + 2 * size_t(it.pointBegin);
            t.pointIndex = it.kind == kTileIndexedPoints
                               ? nullptr
                               : ptr<uint32_t>(b, kSlotPointIndex) + it.pointBegin;
            t.blocks = it.grid.width;
        } else {
            if (!ds_setup(t, lattice, s.ds.fractalDimension, s.ds.scale, s.ds.seed,
                          s.ds.minPixelSize, s.ds.spline, it.grid)) {
                return fail(TG_ERROR_ARGUMENT, "a tile is too coarse for the posts' nodes");
            }
            t.pitch = it.pitch;
        }
        t.postSpacing = P;
        t.heightOffset = it.heightOffset;
        t.status = flags;
        if (it.points) {
            pointFirst.push_back(uint32_t(points));
            points += t.blocks;
            pointJobs.push_back(t);
        } else {
            first.push_back(uint32_t(blocks));
            blocks += t.blocks;
            jobs.push_back(t);
        }
    }
    if (blocks >= 0xffffffffull || points >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "a batch's diamond-square pass holds fewer than 2^32 "
                                          "blocks and points");
    }
    first.push_back(uint32_t(blocks));
    pointFirst.push_back(uint32_t(points));
    for (const auto& [slot, v] : {std::make_pair(kSlotDsJobs, &jobs),
                                  std::make_pair(kSlotDsPointJobs, &pointJobs)}) {
        if (int st = upload(b, slot, v->data(), v->size())) {
            return st;
        }
    }
    for (const auto& [slot, v] : {std::make_pair(kSlotDsFirst, &first),
                                  std::make_pair(kSlotDsPointFirst, &pointFirst)}) {
        if (int st = upload(b, slot, v->data(), v->size())) {
            return st;
        }
    }
    b->dsJobs = uint32_t(jobs.size());
    b->dsBlocks = uint32_t(blocks);
    b->dsPointJobs = uint32_t(pointJobs.size());
    b->dsPoints = uint32_t(points);
    return TG_OK;
}

int load(tg_batch* b, Spec&& spec) {
    if (b->pending) {
        return fail(TG_ERROR_STATE, "the batch's last launch has not finished");
    }
    b->loaded = false;
    b->spec = std::move(spec);
    Spec& s = b->spec;
    // Refs numbered by pairs; the per-octave anchors of grid items (the lattice position of cell
    // (0, 0) split in double, and the lattice steps of a column and a row: Fractal2's rotation and
    // frequency applied to the grid's axes).
    uint64_t rp = 0, bp = 0;
    for (BatchRef& r : s.refs) {
        r.recordPairs = uint32_t(rp);
        r.boulderPairs = uint32_t(bp);
        rp += r.recordCount;
        bp += r.boulderCount;
    }
    if (rp >= 0xffffffffull || bp >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "a batch holds fewer than 2^32 feature pairs");
    }
    b->recordPairs = uint32_t(rp);
    b->boulderPairs = uint32_t(bp);
    const int stride = std::max(s.noise.octaves, 1);
    std::vector<OctaveAnchor> anchors(s.items.size() * size_t(stride));
    size_t outputFloats = 0;
    uint64_t cells = 0;
    for (size_t q = 0; q < s.items.size(); ++q) {
        const Item& it = s.items[q];
        if (it.points) {
            outputFloats = std::max<size_t>(outputFloats, size_t(it.heightOffset) + it.grid.width);
            cells += it.grid.width;
            continue;
        }
        const Grid& g = it.grid;
        outputFloats = std::max(outputFloats, size_t(it.heightOffset) +
                                                  size_t(g.height - 1) * it.pitch + g.width);
        cells += uint64_t(g.width) * g.height;
        const double x0 = g.originX + 0.5 * g.pixelWidth + 0.5 * g.rowRotation;
        const double y0 = g.originY + 0.5 * g.colRotation + 0.5 * g.pixelHeight;
        for (int o = 0; o < s.noise.octaves; ++o) {
            const Octave& oc = s.octaves[size_t(o)];
            const double px = (x0 * oc.tc - y0 * oc.ts) * oc.frequency + oc.ox;
            const double py = (x0 * oc.ts + y0 * oc.tc) * oc.frequency + oc.oy;
            const double fx = std::floor(px), fy = std::floor(py);
            OctaveAnchor& a = anchors[q * size_t(stride) + size_t(o)];
            a.ix = int32_t(uint32_t(uint64_t(int64_t(fx))));
            a.iy = int32_t(uint32_t(uint64_t(int64_t(fy))));
            a.fx = float(px - fx);
            a.fy = float(py - fy);
            a.ax = float(oc.frequency * (g.pixelWidth * oc.tc - g.colRotation * oc.ts));
            a.ay = float(oc.frequency * (g.rowRotation * oc.tc - g.pixelHeight * oc.ts));
            a.bx = float(oc.frequency * (g.pixelWidth * oc.ts + g.colRotation * oc.tc));
            a.by = float(oc.frequency * (g.rowRotation * oc.ts + g.pixelHeight * oc.tc));
        }
    }
    b->outputFloats = outputFloats;
    b->cells = cells;
    if (int st = upload(b, kSlotAnchors, anchors.data(), anchors.size())) {
        return st;
    }
    if (int st = upload(b, kSlotRefs, s.refs.data(), s.refs.size())) {
        return st;
    }
    if (int st = upload(b, kSlotPoints, s.points.data(), s.points.size())) {
        return st;
    }
    if (int st = upload(b, kSlotPointIndex, s.pointIndex.data(), s.pointIndex.size())) {
        return st;
    }
    if (int st = upload(b, kSlotPointTable, s.pointTable.data(), s.pointTable.size())) {
        return st;
    }
    if (int st = upload(b, kSlotPointRegions, s.pointRegions.data(), s.pointRegions.size())) {
        return st;
    }
    TG_CUDA(b->slots[kSlotCraterBoxes].reserve(std::max<size_t>(rp, 1) * sizeof(int4)),
            "allocation");
    TG_CUDA(b->slots[kSlotCraterCulls].reserve(std::max<size_t>(rp, 1) * sizeof(float)),
            "allocation");
    TG_CUDA(b->slots[kSlotBoulderWindows].reserve(std::max<size_t>(bp, 1) * sizeof(int4)),
            "allocation");
    TG_CUDA(b->slots[kSlotHeader].reserve(sizeof(BatchHeader)), "allocation");
    if (int st = load_ds(b)) {  // after the points and the header are on the device
        return st;
    }
    if (int st = plan_bins(b)) {
        return st;
    }
    // A first guess at the entries (a few per bin, not above a few per pair); a launch that
    // needs more grows them.
    TG_CUDA(b->slots[kSlotCraterEntries].reserve(
                (std::min<size_t>(size_t(rp) * 4, size_t(b->bins) * 8) + 1024) * sizeof(BinEntry)),
            "allocation");
    TG_CUDA(b->slots[kSlotBoulderEntries].reserve(
                (std::min<size_t>(size_t(bp) * 2, size_t(b->bins) * 4) + 1024) *
                sizeof(BoulderEntry)),
            "allocation");
    b->loaded = true;
    b->last.cells = cells;
    return TG_OK;
}

// The header of a launch into `out` in pinned[0], and the graphs captured for it; `s` its
// signature.
int prepare(tg_batch* b, float* out, Signature& s) {
    BatchHeader h{};
    h.tiles = uint32_t(b->tiles.size());
    h.refs = uint32_t(b->spec.refs.size());
    h.bins = b->bins;
    h.refRecords = b->recordPairs;
    h.refBoulders = b->boulderPairs;
    h.heights = out;
    h.dsJobs = b->dsJobs;
    h.dsBlocks = b->dsBlocks;
    h.dsPointJobs = b->dsPointJobs;
    h.dsPoints = b->dsPoints;
    h.evalEnd = 0xffffffffu;
    b->pinned[0] = h;
    s = signature(b);
    if (b->exec[1] == nullptr || std::memcmp(&s, &b->captured, sizeof(Signature)) != 0) {
        if (int st = capture(b, s)) {
            return st;
        }
    }
    return TG_OK;
}

int launch(tg_batch* b, float* out, cudaStream_t stream) {
    if (b->pending) {
        return fail(TG_ERROR_STATE, "the batch's last launch has not finished");
    }
    Signature s;
    if (int st = prepare(b, out, s)) {
        return st;
    }
    TG_CUDA(cudaEventRecord(b->events[0], stream), "event record");
    TG_CUDA(cudaGraphLaunch(b->exec[0], stream), "graph launch");
    TG_CUDA(cudaEventRecord(b->events[1], stream), "event record");
    TG_CUDA(cudaGraphLaunch(b->exec[1], stream), "graph launch");
    TG_CUDA(cudaEventRecord(b->events[2], stream), "event record");
    ++b->replays;
    b->pending = true;
    b->out = out;
    b->launchStream = stream;
    b->launched = s;
    return TG_OK;
}

// launch() for host heights: the binning graph, then the evaluation by chunks of consecutive
// items in the work queue's order (about equal output each: the queue's cursor and end set per
// chunk), each chunk's items' output ranges (merged where they meet) copied into `heights` on the
// copy stream while the next chunk is evaluated. Pending like launch(); finish() completes it (a
// relaunch for more entries copies nothing).
int launch_chunked(tg_batch* b, float* out, float* heights, cudaStream_t stream) {
    if (b->pending) {
        return fail(TG_ERROR_STATE, "the batch's last launch has not finished");
    }
    if (b->copyStream == nullptr) {
        TG_CUDA(cudaStreamCreateWithFlags(&b->copyStream, cudaStreamNonBlocking), "stream");
        for (cudaEvent_t& e : b->chunkDone) {
            TG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        }
        TG_CUDA(cudaMallocHost(&b->chunkWords, 2 * kOutputChunks * sizeof(uint32_t)),
                "pinned allocation");
    }
    Signature sig;
    if (int st = prepare(b, out, sig)) {
        return st;
    }
    // Each item's output range; chunks cut at about equal shares of the output.
    const size_t items = b->tiles.size();
    std::vector<uint64_t> lo(items), hi(items);
    uint64_t total = 0;
    for (size_t i = 0; i < items; ++i) {
        const Item& it = b->spec.items[i];
        lo[i] = it.heightOffset;
        hi[i] = it.points ? lo[i] + it.grid.width
                          : lo[i] + uint64_t(it.grid.height - 1) * it.pitch + it.grid.width;
        total += hi[i] - lo[i];
    }
    BatchHeader* header = ptr<BatchHeader>(b, kSlotHeader);
    TG_CUDA(cudaEventRecord(b->events[0], stream), "event record");
    TG_CUDA(cudaGraphLaunch(b->exec[0], stream), "graph launch");
    TG_CUDA(cudaEventRecord(b->events[1], stream), "event record");
    size_t first = 0;
    uint64_t covered = 0;
    for (int c = 0; c < kOutputChunks && first < items; ++c) {
        size_t end = first;
        const uint64_t target = total * uint64_t(c + 1) / kOutputChunks;
        while (end < items && (end == first || covered < target || c + 1 == kOutputChunks)) {
            covered += hi[end] - lo[end];
            ++end;
        }
        // The chunk's output ranges in address order, merged across gaps under 16 KB.
        std::vector<std::pair<uint64_t, uint64_t>> ranges;
        for (size_t i = first; i < end; ++i) {
            ranges.emplace_back(lo[i], hi[i]);
        }
        std::sort(ranges.begin(), ranges.end());
        std::vector<std::pair<uint64_t, uint64_t>> merged;
        for (const auto& r : ranges) {
            if (!merged.empty() && r.first <= merged.back().second + 4096) {
                merged.back().second = std::max(merged.back().second, r.second);
            } else {
                merged.push_back(r);
            }
        }
        uint32_t* words = b->chunkWords + 2 * c;
        words[0] = b->tiles[first].binBase;
        words[1] = end < items ? b->tiles[end].binBase : b->bins;
        TG_CUDA(cudaMemcpyAsync(&header->next, &words[0], sizeof(uint32_t),
                                cudaMemcpyHostToDevice, stream),
                "copy to device");
        TG_CUDA(cudaMemcpyAsync(&header->evalEnd, &words[1], sizeof(uint32_t),
                                cudaMemcpyHostToDevice, stream),
                "copy to device");
        TG_CUDA(launch_batch_evaluate(sig.kernel, sig.noise, sig.view, sig.variant, sig.fast,
                                      sig.ctas, stream),
                "evaluation launch");
        TG_CUDA(cudaEventRecord(b->chunkDone[c], stream), "event record");
        TG_CUDA(cudaStreamWaitEvent(b->copyStream, b->chunkDone[c], 0), "stream wait");
        for (const auto& [from, to] : merged) {
            TG_CUDA(cudaMemcpyAsync(heights + from, out + from, (to - from) * sizeof(float),
                                    cudaMemcpyDeviceToHost, b->copyStream),
                    "copy to host");
        }
        first = end;
    }
    TG_CUDA(cudaMemcpyAsync(&b->pinned[1], header, sizeof(BatchHeader), cudaMemcpyDeviceToHost,
                            stream),
            "copy to host");
    // The launch ends when its copies have.
    TG_CUDA(cudaEventRecord(b->chunkDone[0], b->copyStream), "event record");
    TG_CUDA(cudaStreamWaitEvent(stream, b->chunkDone[0], 0), "stream wait");
    TG_CUDA(cudaEventRecord(b->events[2], stream), "event record");
    ++b->replays;
    b->pending = true;
    b->out = out;
    b->launchStream = stream;
    b->launched = sig;
    return TG_OK;
}

bool done(tg_batch* b) {
    return !b->pending || cudaEventQuery(b->events[2]) == cudaSuccess;
}

int finish(tg_batch* b) {
    for (int attempt = 0; attempt < 3; ++attempt) {
        if (!b->pending) {
            return TG_OK;
        }
        TG_CUDA(cudaEventSynchronize(b->events[2]), "synchronize");
        b->pending = false;
        const BatchHeader r = b->pinned[1];
        if (r.flags & 2u) {
            return fail(TG_ERROR_TIMEOUT, "a bin's staged copy did not arrive");
        }
        if (r.flags & 1u) {
            return fail(TG_ERROR_UNSUPPORTED, "crater datums are not supported in batches");
        }
        if ((r.flags & 8u) && b->spec.fast) {
            return fail(TG_ERROR_STATE, "a record needs the general shaping path");
        }
        if (r.flags & 16u) {
            return fail(TG_ERROR_MEMORY, "a diamond-square block outgrew its shared memory");
        }
        b->last.crater_pairs = r.craterPairs;
        b->last.boulder_pairs = r.boulderPairs;
        b->last.crater_entries = r.craterEntries;
        b->last.boulder_entries = r.boulderEntries;
        b->last.ctas = b->launched.ctas;
        TG_CUDA(cudaEventElapsedTime(&b->last.bin_ms, b->events[0], b->events[1]), "elapsed");
        TG_CUDA(cudaEventElapsedTime(&b->last.evaluate_ms, b->events[1], b->events[2]), "elapsed");
        TG_CUDA(cudaEventElapsedTime(&b->last.graph_ms, b->events[0], b->events[2]), "elapsed");
        const bool craterShort = r.craterEntries > b->launched.view.craterCapacity;
        const bool boulderShort = r.boulderEntries > b->launched.view.boulderCapacity;
        if (!craterShort && !boulderShort) {
            return TG_OK;
        }
        if (craterShort) {
            TG_CUDA(b->slots[kSlotCraterEntries].reserve(size_t(r.craterEntries) *
                                                         sizeof(BinEntry)),
                    "allocation");
        }
        if (boulderShort) {
            TG_CUDA(b->slots[kSlotBoulderEntries].reserve(size_t(r.boulderEntries) *
                                                          sizeof(BoulderEntry)),
                    "allocation");
        }
        if (int st = launch(b, b->out, b->launchStream)) {
            return st;
        }
    }
    return fail(TG_ERROR_STATE, "batch entry capacities did not settle");
}

size_t output_floats(const tg_batch* b) {
    return b->outputFloats;
}

uint64_t cells(const tg_batch* b) {
    return b->cells;
}

uint32_t replays(const tg_batch* b) {
    return b->replays;
}

size_t device_bytes(const tg_batch* b) {
    size_t total = 0;
    for (const Buffer& s : b->slots) {
        total += s.bytes;
    }
    return total;
}

}  // namespace batch
}  // namespace tgb

namespace {

int replay(tg_batch* b, float* out, cudaStream_t stream) {
    if (int st = batch::launch(b, out, stream)) {
        return st;
    }
    return batch::finish(b);
}

// A host input's features copied into the batch's own slots.
int upload_features(tg_batch* b, const tg_batch_input* in, Features& f) {
    if (int s = upload(b, kSlotRecords, static_cast<const CraterRecord*>(in->crater_records),
                       in->n_craters)) {
        return s;
    }
    if (in->crater_footprints != nullptr) {
        if (int s = upload(b, kSlotFootprints, in->crater_footprints, size_t(in->n_craters) * 3)) {
            return s;
        }
    }
    if (int s = upload(b, kSlotData, in->crater_data, in->n_crater_data)) {
        return s;
    }
    static_assert(sizeof(tg_boulder) == sizeof(BoulderRecord), "tg_boulder is a BoulderRecord");
    if (int s = upload(b, kSlotBoulders, reinterpret_cast<const BoulderRecord*>(in->boulders),
                       in->n_boulders)) {
        return s;
    }
    TG_CUDA(b->slots[kSlotHarmonics].reserve(std::max<size_t>(in->n_crater_data, 1) *
                                             sizeof(float)),
            "allocation");
    f.records = ptr<CraterRecord>(b, kSlotRecords);
    f.footprints = in->crater_footprints != nullptr ? ptr<double>(b, kSlotFootprints) : nullptr;
    f.data = ptr<float>(b, kSlotData);
    f.harmonics = ptr<float>(b, kSlotHarmonics);
    f.boulders = ptr<BoulderRecord>(b, kSlotBoulders);
    return TG_OK;
}

// Checks a tile's or point set's feature ranges and the data its records read.
int check_ranges(const tg_batch_input* in, uint32_t crater_begin, uint32_t crater_count,
                 uint32_t data_begin, uint32_t boulder_begin, uint32_t boulder_count,
                 double boulder_width, const char* what, uint32_t i) {
    if (uint64_t(crater_begin) + crater_count > in->n_craters ||
        uint64_t(boulder_begin) + boulder_count > in->n_boulders ||
        data_begin > in->n_crater_data) {
        return fail(TG_ERROR_ARGUMENT, "%s %u: ranges outside the batch's arrays", what, i);
    }
    if (!(boulder_width >= 0.0) || !std::isfinite(boulder_width)) {
        return fail(TG_ERROR_ARGUMENT, "%s %u: boulder width must be finite, >= 0", what, i);
    }
    const CraterRecord* records = static_cast<const CraterRecord*>(in->crater_records);
    const uint64_t room = in->n_crater_data - data_begin;
    for (uint32_t r = crater_begin; r < crater_begin + crater_count; ++r) {
        if (uint64_t(records[r].harmonicOffset) + 2ull * records[r].harmonicCount > room ||
            uint64_t(records[r].tableOffset) + records[r].tableCount > room) {
            return fail(TG_ERROR_ARGUMENT, "crater record %u: data outside the batch's", r);
        }
    }
    return TG_OK;
}

}  // namespace

extern "C" {

int tg_batch_create(tg_device* device, tg_batch** batch) {
    if (batch == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "batch is null");
    }
    *batch = nullptr;
    if (int s = check_device(device)) {
        return s;
    }
    tg_batch* b = new tg_batch();
    b->dev = device;
    cudaError_t err = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 3 && err == cudaSuccess; ++i) {
        err = cudaEventCreate(&b->events[i]);
    }
    if (err == cudaSuccess) {
        err = cudaMallocHost(&b->pinned, 2 * sizeof(BatchHeader));
    }
    if (err == cudaSuccess) {
        err = b->slots[kSlotHeader].reserve(sizeof(BatchHeader));
    }
    if (err != cudaSuccess) {
        tg_batch_destroy(b);
        return cuda_fail(err, "batch set-up");
    }
    std::memset(b->pinned, 0, 2 * sizeof(BatchHeader));
    *batch = b;
    return TG_OK;
}

void tg_batch_destroy(tg_batch* b) {
    if (b == nullptr) {
        return;
    }
    if (b->dev != nullptr) {
        cudaSetDevice(b->dev->ordinal);
    }
    if (b->pending) {
        cudaEventSynchronize(b->events[2]);
    }
    if (b->stream != nullptr) {
        cudaStreamSynchronize(b->stream);
    }
    drop_graph(b);
    for (Buffer& s : b->slots) {
        s.release();
    }
    for (cudaEvent_t e : b->events) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    if (b->pinned != nullptr) {
        cudaFreeHost(b->pinned);
    }
    if (b->chunkWords != nullptr) {
        cudaFreeHost(b->chunkWords);
    }
    for (cudaEvent_t e : b->chunkDone) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    if (b->copyStream != nullptr) {
        cudaStreamSynchronize(b->copyStream);
        cudaStreamDestroy(b->copyStream);
    }
    if (b->stream != nullptr) {
        cudaStreamDestroy(b->stream);
    }
    delete b;
}

int tg_batch_load(tg_batch* b, const tg_batch_input* in) {
    if (int s = check_batch(b)) {
        return s;
    }
    if (in == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "input is null");
    }
    if (b->pending) {
        return fail(TG_ERROR_STATE, "the batch's last launch has not finished");
    }
    b->loaded = false;
    if ((in->n_tiles > 0 && in->tiles == nullptr) ||
        (in->n_fractals > 0 && in->fractals == nullptr) ||
        (in->n_craters > 0 && (in->crater_records == nullptr || in->crater_kernel == nullptr)) ||
        (in->n_crater_data > 0 && in->crater_data == nullptr) ||
        (in->n_boulders > 0 && in->boulders == nullptr) ||
        (in->n_point_sets > 0 && in->point_sets == nullptr) ||
        (in->n_points > 0 && in->points == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "a batch input array is null");
    }
    Spec spec;
    if (int s = make_noise(in->fractals, in->n_fractals, in->elevation, spec.noise,
                           spec.octaves)) {
        return s;
    }
    // Craters: one kernel for every item; datums are refused, features beyond outlines take the
    // general shaping path.
    if (in->crater_kernel != nullptr) {
        std::memcpy(&spec.kernel, in->crater_kernel, sizeof(spec.kernel));
    }
    const CraterRecord* records = static_cast<const CraterRecord*>(in->crater_records);
    uint32_t heavy = 0;
    for (uint32_t i = 0; i < in->n_craters; ++i) {
        const CraterRecord& r = records[i];
        if (r.hasDatum == 1u) {
            return fail(TG_ERROR_UNSUPPORTED, "crater datums are not supported in batches");
        }
        if (r.tableCount > 0u || r.markCount > 0u || r.terraceCount > 0u || r.peakCount > 0u ||
            r.shiftX != 0.0f || r.shiftY != 0.0f || r.upslopeX != 0.0f || r.upslopeY != 0.0f) {
            heavy = 4u;
        }
    }
    spec.fast = crater_fast_path(spec.kernel, heavy);

    // Tiles: checked, empty ones dropped, queued coarsest spacing first (their bins hold the
    // most entries), then largest first; point sets after them.
    std::vector<uint32_t> order;
    for (uint32_t i = 0; i < in->n_tiles; ++i) {
        const tg_tile& t = in->tiles[i];
        Grid g;
        if (int s = to_grid(&t.grid, g)) {
            return s;
        }
        if (t.pitch < t.grid.width) {
            return fail(TG_ERROR_ARGUMENT, "tile %u: pitch below its width", i);
        }
        if (int s = check_ranges(in, t.crater_begin, t.crater_count, t.data_begin,
                                 t.boulder_begin, t.boulder_count, t.boulder_width, "tile", i)) {
            return s;
        }
        if (uint64_t(t.grid.width) * t.grid.height > 0) {
            order.push_back(i);
        }
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) {
        const tg_grid& ga = in->tiles[a].grid;
        const tg_grid& gc = in->tiles[c].grid;
        const double sa = std::fabs(ga.pixel_width * ga.pixel_height);
        const double sc = std::fabs(gc.pixel_width * gc.pixel_height);
        if (sa != sc) {
            return sa > sc;
        }
        return uint64_t(ga.width) * ga.height > uint64_t(gc.width) * gc.height;
    });
    for (uint32_t i : order) {
        const tg_tile& t = in->tiles[i];
        Item it{};
        to_grid(&t.grid, it.grid);
        it.heightOffset = t.height_offset;
        it.pitch = t.pitch;
        it.points = false;
        it.kind = kTileGrid;
        it.pointBegin = kNone;
        it.boulderWidth = t.boulder_width;
        spec.refs.push_back(BatchRef{uint32_t(spec.items.size()), t.crater_begin, t.crater_count,
                                     t.data_begin, t.boulder_begin, t.boulder_count, 0, 0});
        spec.items.push_back(it);
    }
    for (uint32_t i = 0; i < in->n_point_sets; ++i) {
        const tg_point_set& p = in->point_sets[i];
        if (uint64_t(p.point_begin) + p.point_count > in->n_points) {
            return fail(TG_ERROR_ARGUMENT, "point set %u: points outside the batch's", i);
        }
        if (int s = check_ranges(in, p.crater_begin, p.crater_count, p.data_begin,
                                 p.boulder_begin, p.boulder_count, p.boulder_width, "point set",
                                 i)) {
            return s;
        }
        for (uint32_t q = p.point_begin; q < p.point_begin + p.point_count; ++q) {
            if (!std::isfinite(in->points[2 * size_t(q)]) ||
                !std::isfinite(in->points[2 * size_t(q) + 1])) {
                return fail(TG_ERROR_ARGUMENT, "point set %u: a point is not finite", i);
            }
        }
        if (p.point_count == 0) {
            continue;
        }
        Item it{};
        it.grid = Grid{p.point_count, 1, 0.0, 1.0, 0.0, 0.0, 0.0, -1.0};
        it.heightOffset = p.height_offset;
        it.pitch = p.point_count;
        it.points = true;
        it.kind = kTilePoints;
        it.pointBegin = uint32_t(spec.pointIndex.size());
        it.boulderWidth = p.boulder_width;
        append_points(spec, in->points + 2 * size_t(p.point_begin), p.point_count);
        spec.refs.push_back(BatchRef{uint32_t(spec.items.size()), p.crater_begin, p.crater_count,
                                     p.data_begin, p.boulder_begin, p.boulder_count, 0, 0});
        spec.items.push_back(it);
    }
    if (int s = upload_features(b, in, spec.features)) {
        return s;
    }
    return load(b, std::move(spec));
}

int tg_batch_evaluate(tg_batch* b, float* heights, size_t n_heights, int memory, void* stream) {
    if (int s = check_batch(b)) {
        return s;
    }
    if (!b->loaded) {
        return fail(TG_ERROR_STATE, "no batch is loaded");
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (n_heights < b->outputFloats || (b->outputFloats > 0 && heights == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "the batch writes %zu floats", b->outputFloats);
    }
    if (b->tiles.empty()) {
        return TG_OK;
    }
    float* out = heights;
    cudaStream_t s = b->stream;
    if (memory == TG_MEMORY_DEVICE) {
        if (reinterpret_cast<uintptr_t>(heights) % sizeof(float) != 0) {
            return fail(TG_ERROR_ARGUMENT, "heights must be 4-byte aligned");
        }
        if (stream != nullptr) {
            s = static_cast<cudaStream_t>(stream);
        }
    } else {
        TG_CUDA(b->slots[kSlotOutput].reserve(b->outputFloats * sizeof(float)), "allocation");
        out = ptr<float>(b, kSlotOutput);
    }
    cudaPointerAttributes where{};
    const bool pinned = memory == TG_MEMORY_HOST &&
                        cudaPointerGetAttributes(&where, heights) == cudaSuccess &&
                        where.type == cudaMemoryTypeHost;
    (void)cudaGetLastError();
    if (pinned && !b->spec.ds.on && b->tiles.size() >= 2) {
        // Page-locked heights cross to the host chunk by chunk while later chunks are evaluated;
        // if the bins needed more entries, the batch ran again whole and its heights are copied
        // again.
        const uint32_t before = b->replays;
        if (int st = launch_chunked(b, out, heights, s)) {
            return st;
        }
        if (int st = finish(b)) {
            return st;
        }
        if (b->replays == before + 1) {
            return TG_OK;
        }
    } else if (int st = replay(b, out, s)) {
        return st;
    }
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(cudaMemcpyAsync(heights, out, b->outputFloats * sizeof(float),
                                cudaMemcpyDeviceToHost, s),
                "copy to host");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    }
    return TG_OK;
}

int tg_batch_run(tg_batch* b, const tg_batch_input* in, float* heights, size_t n_heights,
                 int memory, void* stream) {
    if (int s = tg_batch_load(b, in)) {
        return s;
    }
    return tg_batch_evaluate(b, heights, n_heights, memory, stream);
}

int tg_batch_variant_count(void) {
    return batch_variant_count();
}

int tg_batch_variant(int index, uint32_t* bin_width, uint32_t* bin_height,
                     uint32_t* cells_per_thread) {
    if (index < 0 || index >= batch_variant_count()) {
        return fail(TG_ERROR_ARGUMENT, "variant %d of %d", index, batch_variant_count());
    }
    const BatchVariant v = batch_variant(index);
    if (bin_width != nullptr) {
        *bin_width = v.binW;
    }
    if (bin_height != nullptr) {
        *bin_height = v.binH;
    }
    if (cells_per_thread != nullptr) {
        *cells_per_thread = v.cellsPerThread;
    }
    return TG_OK;
}

int tg_batch_set_variant(tg_batch* b, int index) {
    if (int s = check_batch(b)) {
        return s;
    }
    if (index < 0 || index >= batch_variant_count()) {
        return fail(TG_ERROR_ARGUMENT, "variant %d of %d", index, batch_variant_count());
    }
    if (b->pending) {
        return fail(TG_ERROR_STATE, "the batch's last launch has not finished");
    }
    b->variant = index;
    return b->loaded ? plan_bins(b) : TG_OK;
}

int tg_batch_tune(tg_batch* b, int trials, float* ms) {
    if (int s = check_batch(b)) {
        return s;
    }
    if (!b->loaded) {
        return fail(TG_ERROR_STATE, "no batch is loaded");
    }
    if (trials < 1) {
        return fail(TG_ERROR_ARGUMENT, "trials must be at least 1");
    }
    if (b->tiles.empty()) {
        return TG_OK;
    }
    TG_CUDA(b->slots[kSlotOutput].reserve(b->outputFloats * sizeof(float)), "allocation");
    float* out = ptr<float>(b, kSlotOutput);
    const int count = batch_variant_count();
    int best = 0;
    float bestMs = INFINITY;
    for (int v = 0; v < count; ++v) {
        float median = NAN;
        if (b->spec.fast || v == 0) {
            b->variant = v;
            if (int s = plan_bins(b)) {
                return s;
            }
            if (int s = replay(b, out, b->stream)) {  // warm-up, capture, entry sizing
                return s;
            }
            std::vector<float> times;
            for (int t = 0; t < trials; ++t) {
                if (int s = replay(b, out, b->stream)) {
                    return s;
                }
                times.push_back(b->last.graph_ms);
            }
            std::sort(times.begin(), times.end());
            median = times[times.size() / 2];
            if (median < bestMs) {
                bestMs = median;
                best = v;
            }
        }
        if (ms != nullptr) {
            ms[v] = median;
        }
    }
    b->variant = best;
    return plan_bins(b);
}

int tg_batch_stats_get(tg_batch* b, tg_batch_stats* stats) {
    if (b == nullptr || stats == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "batch and stats are required");
    }
    tg_batch_stats s = b->last;
    const int v = effective_variant(b);
    const BatchVariant shape = batch_variant(v);
    s.variant = uint32_t(v);
    s.bin_width = shape.binW;
    s.bin_height = shape.binH;
    s.cells_per_thread = shape.cellsPerThread;
    s.fast = b->spec.fast ? 1u : 0u;
    s.bins = b->bins;
    s.cells = b->cells;
    s.captures = b->captures;
    s.replays = b->replays;
    *stats = s;
    return TG_OK;
}

}  // extern "C"
