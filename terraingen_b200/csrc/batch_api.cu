// The batched form's C ABI (tg_batch_* in include/tgb200.h): input checks, the per-tile lattice
// anchors (double), the tiles' bin numbering and queue order, device buffers sized by capacity,
// CUDA graph capture and replay, and the autotuner over kernel shapes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "kernels.h"

using namespace tgb;
using namespace tgb::api;

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

// The octaves of a Perlin fBm: what every cell shares (float, as Fractal2 accumulates them) and
// what the per-tile anchors need in double.
struct Octave {
    double frequency, tc, ts, ox, oy;
};

enum BatchSlot {
    kSlotTiles,
    kSlotAnchors,
    kSlotRecords,
    kSlotRecordTile,
    kSlotFootprints,
    kSlotData,
    kSlotHarmonics,
    kSlotBoulders,
    kSlotBoulderTile,
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
    kSlotBatchSlots
};

// What a captured graph depends on; a change means a new capture.
struct Signature {
    BatchView view;
    int variant;
    bool fast;
    uint32_t ctas, maxRecords, maxBoulders;
    CraterShapeKernel kernel;
    BatchNoise noise;
};

}  // namespace

struct tg_batch {
    tg_device* dev = nullptr;
    cudaStream_t stream = nullptr;
    // Recorded before the binning graph, between it and the evaluation graph, and after.
    cudaEvent_t events[3] = {nullptr, nullptr, nullptr};
    BatchHeader* pinned = nullptr;  // [0] written before each replay, [1] read back after
    Buffer slots[kSlotBatchSlots];
    int variant = 0;

    // The loaded batch.
    bool loaded = false;
    std::vector<tg_tile> tiles;  // queue order
    std::vector<OctaveAnchor> anchors;
    BatchNoise noise{};
    CraterShapeKernel kernel{};
    bool fast = true;
    uint32_t records = 0, boulders = 0, nData = 0;
    bool footprints = false;
    size_t outputFloats = 0;
    uint64_t cells = 0;
    uint32_t bins = 0;

    // Graph state.
    cudaGraph_t graph[2] = {nullptr, nullptr};  // binning, evaluation
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
    return b->fast ? b->variant : 0;
}

// Numbers the loaded tiles' bins for the current kernel shape and uploads the tile table.
int plan_bins(tg_batch* b) {
    const BatchVariant v = batch_variant(effective_variant(b));
    std::vector<BatchTile> out(b->tiles.size());
    uint64_t base = 0;
    for (size_t i = 0; i < b->tiles.size(); ++i) {
        const tg_tile& t = b->tiles[i];
        BatchTile& d = out[i];
        d.grid = Grid{t.grid.width,        t.grid.height,       t.grid.origin_x,
                      t.grid.pixel_width,  t.grid.row_rotation, t.grid.origin_y,
                      t.grid.col_rotation, t.grid.pixel_height};
        d.heightOffset = t.height_offset;
        d.pitch = t.pitch;
        d.binsX = (t.grid.width + v.binW - 1) / v.binW;
        d.binsY = (t.grid.height + v.binH - 1) / v.binH;
        d.binBase = uint32_t(base);
        d.dataBase = t.data_begin;
        d.anchorBase = uint32_t(i) * uint32_t(std::max(b->noise.octaves, 1));
        d.boulderWidth = t.boulder_width;
        base += uint64_t(d.binsX) * d.binsY;
    }
    if (base >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "a batch holds fewer than 2^32 bins");
    }
    b->bins = uint32_t(base);
    const size_t words = size_t(b->bins) + 1;
    TG_CUDA(b->slots[kSlotCraterCounts].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotCraterCursor].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotBoulderCounts].reserve(words * sizeof(uint32_t)), "allocation");
    TG_CUDA(b->slots[kSlotBoulderCursor].reserve(words * sizeof(uint32_t)), "allocation");
    const uint32_t capBins =
        std::min(capacity<uint32_t>(b, kSlotCraterCounts), capacity<uint32_t>(b, kSlotBoulderCounts)) - 1;
    TG_CUDA(b->slots[kSlotScanScratch].reserve(scan_scratch_words(capBins) * sizeof(uint32_t)),
            "allocation");
    if (!out.empty()) {
        TG_CUDA(b->slots[kSlotTiles].reserve(out.size() * sizeof(BatchTile)), "allocation");
        TG_CUDA(cudaMemcpyAsync(b->slots[kSlotTiles].ptr, out.data(), out.size() * sizeof(BatchTile),
                                cudaMemcpyHostToDevice, b->stream),
                "copy to device");
    }
    TG_CUDA(cudaStreamSynchronize(b->stream), "synchronize");
    return TG_OK;
}

BatchView make_view(tg_batch* b) {
    BatchView v{};
    v.header = ptr<BatchHeader>(b, kSlotHeader);
    v.tiles = ptr<BatchTile>(b, kSlotTiles);
    v.anchors = ptr<OctaveAnchor>(b, kSlotAnchors);
    v.records = ptr<CraterRecord>(b, kSlotRecords);
    v.recordTile = ptr<uint32_t>(b, kSlotRecordTile);
    v.footprints = b->footprints ? ptr<double>(b, kSlotFootprints) : nullptr;
    v.data = ptr<float>(b, kSlotData);
    v.harmonics = ptr<float>(b, kSlotHarmonics);
    v.boulders = ptr<BoulderRecord>(b, kSlotBoulders);
    v.boulderTile = ptr<uint32_t>(b, kSlotBoulderTile);
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
    v.capacityBins =
        std::min(capacity<uint32_t>(b, kSlotCraterCounts), capacity<uint32_t>(b, kSlotBoulderCounts)) - 1;
    return v;
}

Signature signature(tg_batch* b) {
    Signature s;
    std::memset(&s, 0, sizeof(s));
    s.view = make_view(b);
    s.variant = effective_variant(b);
    s.fast = b->fast;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev->ordinal);
    s.ctas = uint32_t(sms * batch_blocks_per_sm(s.variant, b->fast));
    s.maxRecords = std::min(capacity<CraterRecord>(b, kSlotRecords), capacity<uint32_t>(b, kSlotRecordTile));
    s.maxBoulders =
        std::min(capacity<BoulderRecord>(b, kSlotBoulders), capacity<uint32_t>(b, kSlotBoulderTile));
    s.kernel = b->kernel;
    s.noise = b->noise;
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
        err = launch_batch_bin(s.kernel, s.view, batch_variant(s.variant), s.maxRecords,
                               s.maxBoulders, ptr<uint32_t>(b, kSlotScanScratch), b->stream);
    }
    if (int st = finish_capture(b, 0, err)) {
        return st;
    }
    TG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    err = launch_batch_evaluate(s.kernel, s.noise, s.view, s.variant, s.fast, s.ctas, b->stream);
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

// One replay of the loaded batch into `out` on `stream`, growing the entry capacities (and
// re-capturing) when the bins needed more than they held.
int replay(tg_batch* b, float* out, cudaStream_t stream) {
    for (int attempt = 0; attempt < 3; ++attempt) {
        BatchHeader h{};
        h.tiles = uint32_t(b->tiles.size());
        h.records = b->records;
        h.boulders = b->boulders;
        h.bins = b->bins;
        h.heights = out;
        b->pinned[0] = h;
        const Signature s = signature(b);
        if (b->exec[1] == nullptr || std::memcmp(&s, &b->captured, sizeof(Signature)) != 0) {
            if (int st = capture(b, s)) {
                return st;
            }
        }
        TG_CUDA(cudaEventRecord(b->events[0], stream), "event record");
        TG_CUDA(cudaGraphLaunch(b->exec[0], stream), "graph launch");
        TG_CUDA(cudaEventRecord(b->events[1], stream), "event record");
        TG_CUDA(cudaGraphLaunch(b->exec[1], stream), "graph launch");
        TG_CUDA(cudaEventRecord(b->events[2], stream), "event record");
        ++b->replays;
        TG_CUDA(cudaStreamSynchronize(stream), "synchronize");
        const BatchHeader r = b->pinned[1];
        if (r.flags & 2u) {
            return fail(TG_ERROR_TIMEOUT, "a bin's staged copy did not arrive");
        }
        if (r.flags & 1u) {
            return fail(TG_ERROR_UNSUPPORTED, "crater datums are not supported in batches");
        }
        if ((r.flags & 8u) && b->fast) {
            return fail(TG_ERROR_STATE, "a record needs the general shaping path");
        }
        const bool craterShort = r.craterEntries > s.view.craterCapacity;
        const bool boulderShort = r.boulderEntries > s.view.boulderCapacity;
        b->last.crater_pairs = r.craterPairs;
        b->last.boulder_pairs = r.boulderPairs;
        b->last.crater_entries = r.craterEntries;
        b->last.boulder_entries = r.boulderEntries;
        b->last.ctas = s.ctas;
        TG_CUDA(cudaEventElapsedTime(&b->last.bin_ms, b->events[0], b->events[1]), "elapsed");
        TG_CUDA(cudaEventElapsedTime(&b->last.evaluate_ms, b->events[1], b->events[2]), "elapsed");
        TG_CUDA(cudaEventElapsedTime(&b->last.graph_ms, b->events[0], b->events[2]), "elapsed");
        if (!craterShort && !boulderShort) {
            return TG_OK;
        }
        if (craterShort) {
            TG_CUDA(b->slots[kSlotCraterEntries].reserve(size_t(r.craterEntries) * sizeof(BinEntry)),
                    "allocation");
        }
        if (boulderShort) {
            TG_CUDA(b->slots[kSlotBoulderEntries].reserve(size_t(r.boulderEntries) *
                                                      sizeof(BoulderEntry)),
                    "allocation");
        }
    }
    return fail(TG_ERROR_STATE, "batch entry capacities did not settle");
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

int check_batch(tg_batch* b) {
    if (b == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "batch is null");
    }
    return check_device(b->dev);
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
    b->loaded = false;
    if ((in->n_tiles > 0 && in->tiles == nullptr) ||
        (in->n_fractals > 0 && in->fractals == nullptr) ||
        (in->n_craters > 0 && (in->crater_records == nullptr || in->crater_kernel == nullptr)) ||
        (in->n_crater_data > 0 && in->crater_data == nullptr) ||
        (in->n_boulders > 0 && in->boulders == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "a batch input array is null");
    }

    // The source: at most one enabled fractal, a Perlin fBm without warp (fractal.h:219-240).
    BatchNoise noise{};
    noise.elevation = in->elevation;
    noise.total = 1.0f;
    std::vector<Octave> octaves;
    const Fractal* only = nullptr;
    for (uint32_t i = 0; i < in->n_fractals; ++i) {
        const Fractal* f = static_cast<const Fractal*>(in->fractals) + i;
        if (!f->enabled) {
            continue;
        }
        if (only != nullptr) {
            return fail(TG_ERROR_UNSUPPORTED, "a batch's source is one fractal");
        }
        only = f;
    }
    if (only != nullptr) {
        if (only->basis != kBasisPerlin || only->type != kTypeFbm ||
            only->warpAmplitude > 0.0f) {
            return fail(TG_ERROR_UNSUPPORTED, "a batch's source is a Perlin fBm without warp");
        }
        if (only->octaves < 1 || only->octaves > kBatchMaxOctaves || !(only->wavelength > 0.0f) ||
            !(only->lacunarity > 1.0f) || !(only->gain > 0.0f)) {
            return fail(TG_ERROR_ARGUMENT, "the fractal is invalid");
        }
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
            frequency *= double(only->lacunarity);
            const double c = double(kTurnCos), s = double(kTurnSin);
            const double nc = tc * c - ts * s;
            ts = ts * c + tc * s;
            tc = nc;
        }
        noise.total = total;
    }

    // Craters: one kernel for every tile; datums are refused, features beyond outlines take the
    // general shaping path.
    CraterShapeKernel kernel{};
    if (in->crater_kernel != nullptr) {
        std::memcpy(&kernel, in->crater_kernel, sizeof(kernel));
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

    // Tiles: checked, empty ones dropped, queued coarsest spacing first (their bins hold the
    // most entries), then largest first.
    std::vector<uint32_t> order;
    size_t outputFloats = 0;
    uint64_t cells = 0;
    std::vector<uint32_t> recordTile(in->n_craters, kNone), boulderTile(in->n_boulders, kNone);
    for (uint32_t i = 0; i < in->n_tiles; ++i) {
        const tg_tile& t = in->tiles[i];
        Grid g;
        if (int s = to_grid(&t.grid, g)) {
            return s;
        }
        if (t.pitch < t.grid.width) {
            return fail(TG_ERROR_ARGUMENT, "tile %u: pitch below its width", i);
        }
        if (uint64_t(t.crater_begin) + t.crater_count > in->n_craters ||
            uint64_t(t.boulder_begin) + t.boulder_count > in->n_boulders ||
            t.data_begin > in->n_crater_data) {
            return fail(TG_ERROR_ARGUMENT, "tile %u: ranges outside the batch's arrays", i);
        }
        if (!(t.boulder_width >= 0.0) || !std::isfinite(t.boulder_width)) {
            return fail(TG_ERROR_ARGUMENT, "tile %u: boulder width must be finite, >= 0", i);
        }
        const uint64_t n = uint64_t(t.grid.width) * t.grid.height;
        if (n == 0) {
            continue;
        }
        const size_t end = size_t(t.height_offset) + size_t(t.grid.height - 1) * t.pitch +
                           t.grid.width;
        outputFloats = std::max(outputFloats, end);
        cells += n;
        order.push_back(i);
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
    const uint32_t available = in->n_crater_data;
    for (uint32_t q = 0; q < order.size(); ++q) {
        const tg_tile& t = in->tiles[order[q]];
        for (uint32_t i = t.crater_begin; i < t.crater_begin + t.crater_count; ++i) {
            if (recordTile[i] != kNone) {
                return fail(TG_ERROR_ARGUMENT, "crater record %u belongs to two tiles", i);
            }
            const CraterRecord& r = records[i];
            const uint64_t room = available - t.data_begin;
            if (uint64_t(r.harmonicOffset) + 2ull * r.harmonicCount > room ||
                uint64_t(r.tableOffset) + r.tableCount > room) {
                return fail(TG_ERROR_ARGUMENT, "crater record %u: data outside the batch's", i);
            }
            recordTile[i] = q;
        }
        for (uint32_t i = t.boulder_begin; i < t.boulder_begin + t.boulder_count; ++i) {
            if (boulderTile[i] != kNone) {
                return fail(TG_ERROR_ARGUMENT, "boulder %u belongs to two tiles", i);
            }
            boulderTile[i] = q;
        }
    }

    // Per tile and octave, the lattice position of cell (0, 0) split in double, and the lattice
    // steps of a column and a row (the rotation and frequency of Fractal2 applied to the grid's
    // axes).
    const int stride = std::max(noise.octaves, 1);
    std::vector<OctaveAnchor> anchors(order.size() * size_t(stride));
    for (size_t q = 0; q < order.size(); ++q) {
        const tg_grid& g = in->tiles[order[q]].grid;
        const double x0 = g.origin_x + 0.5 * g.pixel_width + 0.5 * g.row_rotation;
        const double y0 = g.origin_y + 0.5 * g.col_rotation + 0.5 * g.pixel_height;
        for (int o = 0; o < noise.octaves; ++o) {
            const Octave& oc = octaves[size_t(o)];
            const double px = (x0 * oc.tc - y0 * oc.ts) * oc.frequency + oc.ox;
            const double py = (x0 * oc.ts + y0 * oc.tc) * oc.frequency + oc.oy;
            const double fx = std::floor(px), fy = std::floor(py);
            OctaveAnchor& a = anchors[q * size_t(stride) + size_t(o)];
            a.ix = int32_t(uint32_t(uint64_t(int64_t(fx))));
            a.iy = int32_t(uint32_t(uint64_t(int64_t(fy))));
            a.fx = float(px - fx);
            a.fy = float(py - fy);
            a.ax = float(oc.frequency * (g.pixel_width * oc.tc - g.col_rotation * oc.ts));
            a.ay = float(oc.frequency * (g.row_rotation * oc.tc - g.pixel_height * oc.ts));
            a.bx = float(oc.frequency * (g.pixel_width * oc.ts + g.col_rotation * oc.tc));
            a.by = float(oc.frequency * (g.row_rotation * oc.ts + g.pixel_height * oc.tc));
        }
    }

    // Device copies.
    b->tiles.clear();
    for (uint32_t i : order) {
        b->tiles.push_back(in->tiles[i]);
    }
    b->anchors = anchors;
    b->noise = noise;
    b->kernel = kernel;
    b->fast = crater_fast_path(kernel, heavy);
    b->records = in->n_craters;
    b->boulders = in->n_boulders;
    b->nData = in->n_crater_data;
    b->footprints = in->crater_footprints != nullptr;
    b->outputFloats = outputFloats;
    b->cells = cells;
    if (int s = upload(b, kSlotAnchors, anchors.data(), anchors.size())) {
        return s;
    }
    if (int s = upload(b, kSlotRecords, records, in->n_craters)) {
        return s;
    }
    if (int s = upload(b, kSlotRecordTile, recordTile.data(), recordTile.size())) {
        return s;
    }
    if (b->footprints) {
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
    if (int s = upload(b, kSlotBoulderTile, boulderTile.data(), boulderTile.size())) {
        return s;
    }
    TG_CUDA(b->slots[kSlotHarmonics].reserve(std::max<size_t>(in->n_crater_data, 1) * sizeof(float)),
            "allocation");
    TG_CUDA(b->slots[kSlotCraterBoxes].reserve(std::max<size_t>(in->n_craters, 1) * sizeof(int4)),
            "allocation");
    TG_CUDA(b->slots[kSlotCraterCulls].reserve(std::max<size_t>(in->n_craters, 1) * sizeof(float)),
            "allocation");
    TG_CUDA(b->slots[kSlotBoulderWindows].reserve(std::max<size_t>(in->n_boulders, 1) * sizeof(int4)),
            "allocation");
    // A first guess at the entries (a few bins per record); a replay that needs more grows them.
    TG_CUDA(b->slots[kSlotCraterEntries].reserve((size_t(in->n_craters) * 4 + 64) * sizeof(BinEntry)),
            "allocation");
    TG_CUDA(b->slots[kSlotBoulderEntries].reserve((size_t(in->n_boulders) * 2 + 64) *
                                              sizeof(BoulderEntry)),
            "allocation");
    if (int s = plan_bins(b)) {
        return s;
    }
    b->loaded = true;
    b->last.cells = cells;
    return TG_OK;
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
        if (stream != nullptr) {
            s = static_cast<cudaStream_t>(stream);
        }
    } else {
        TG_CUDA(b->slots[kSlotOutput].reserve(b->outputFloats * sizeof(float)), "allocation");
        out = ptr<float>(b, kSlotOutput);
    }
    if (int st = replay(b, out, s)) {
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
        if (b->fast || v == 0) {
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
    s.fast = b->fast ? 1u : 0u;
    s.bins = b->bins;
    s.cells = b->cells;
    s.captures = b->captures;
    s.replays = b->replays;
    *stats = s;
    return TG_OK;
}

}  // extern "C"
