// The request server (tg_server_* in include/tgb200.h): continuous batching of tile and
// point-query requests over the batch engine (batch_internal.h), feature regions resident in
// device arenas with least-recently-used eviction, and admission by a device memory budget.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "batch_internal.h"
#include "kernels.h"

using namespace tgb;
using namespace tgb::api;

namespace {

struct RegionKey {
    int32_t lod;
    int64_t ix, iy;
    bool operator==(const RegionKey& o) const {
        return lod == o.lod && ix == o.ix && iy == o.iy;
    }
};

struct RegionHash {
    size_t operator()(const RegionKey& k) const {
        uint64_t h = uint64_t(k.lod) * 0x9E3779B97F4A7C15ull;
        h ^= uint64_t(k.ix) + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h ^= uint64_t(k.iy) + 0x85EBCA77C2B2AE63ull + (h << 6) + (h >> 2);
        return size_t(h);
    }
};

// A feature region resident on the device: its records (with footprints) and data in the arenas.
struct Region {
    uint32_t recBegin = 0, recCount = 0;  // owned records (tiles read these)
    uint32_t recTotal = 0;                // owned, then the others reaching in (indexed points)
    uint32_t dataBegin = 0, dataCount = 0;
    uint32_t listBegin = 0, listCount = 0;  // the cell lists (0 when not indexed)
    PointRegion index{};
    uint64_t lastUse = 0;
    uint32_t inFlight = 0;  // batches in flight that read it
};

// First-fit ranges of an arena, in elements.
class Ranges {
public:
    void reset(size_t capacity) {
        free_.clear();
        if (capacity > 0) {
            free_[0] = capacity;
        }
    }
    bool take(size_t n, size_t& at) {
        if (n == 0) {
            at = 0;
            return true;
        }
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                at = it->first;
                const size_t rest = it->second - n;
                free_.erase(it);
                if (rest > 0) {
                    free_[at + n] = rest;
                }
                return true;
            }
        }
        return false;
    }
    void give(size_t at, size_t n) {
        if (n == 0) {
            return;
        }
        auto next = free_.lower_bound(at);
        if (next != free_.end() && at + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == at) {
                prev->second += n;
                return;
            }
        }
        free_[at] = n;
    }

private:
    std::map<size_t, size_t> free_;
};

struct Pending {
    tg_request req;
    bool pinned = false;  // host heights in page-locked memory: copied into directly
    std::vector<double> xy;
    int lod = 0;
    uint64_t cells = 0;
    std::vector<RegionKey> keys;  // the regions whose craters can reach it
    int64_t ix0 = 0, iy0 = 0;     // points: the regions covering their bounding box
    uint32_t tw = 0, th = 0;
    std::vector<uint8_t> occupied;  // points: regions holding a point, tw x th
};

// A region's records built on the host, waiting to be copied into the arenas.
struct Built {
    RegionKey key;
    int status = TG_OK;
    std::vector<CraterRecord> records;  // owned first
    std::vector<double> footprints;
    std::vector<float> culls;
    std::vector<float> data;
    uint32_t owned = 0;
    std::vector<uint32_t> lists;        // the cell lists (indexed regions)
    PointRegion index{};
    bool heavy = false;
    double ms = 0.0;
};

constexpr uint32_t kIndexCells = 16;  // cells across an indexed region

// The cull distance of a record (as the device's crater_reach computes it): beyond it no cell
// is within the crater's reach.
float cull_of(const CraterRecord& r, const float* data, float reachRadii) {
    double sum = 1.0;
    if (r.tableCount > 0u) {
        for (uint32_t n = 0; n < r.tableCount; ++n) {
            sum = std::fmax(sum, 1.0 + double(data[r.tableOffset + n]));
        }
    } else {
        for (uint32_t n = 0; n < r.harmonicCount; ++n) {
            sum += std::fabs(double(data[r.harmonicOffset + 2u * n]));
        }
    }
    const double scale = std::sqrt(double(r.ellipticity)) * sum;
    const bool stretched = r.markCount > 0u || r.terraceCount > 0u || r.shiftX != 0.0f ||
                           r.shiftY != 0.0f;
    return stretched ? INFINITY
                     : float(scale * double(reachRadii) * (0.5 * double(r.diameter)) *
                             (1.0 + 1e-5)) + 1e-6f;
}

// Builds regions' crater records on host worker threads: tg_crater_batch over the region's
// grid, then the craters whose centers lie in the region.
class Builders {
public:
    void start(unsigned n, const tg_server_options& opt, int pointLevel) {
        opt_ = opt;
        pointLevel_ = pointLevel;
        for (unsigned i = 0; i < n; ++i) {
            threads_.emplace_back([this] { work(); });
        }
    }
    void stop() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stopping_ = true;
        }
        wake_.notify_all();
        for (std::thread& t : threads_) {
            t.join();
        }
        threads_.clear();
    }
    void request(const RegionKey& k) {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            if (!asked_.insert(k).second) {
                return;
            }
            jobs_.push_back(k);
        }
        wake_.notify_one();
    }
    std::vector<Built> take() {
        std::lock_guard<std::mutex> lock(mutex_);
        std::vector<Built> out;
        out.swap(done_);
        for (const Built& b : out) {
            asked_.erase(b.key);
        }
        return out;
    }
    bool busy() {
        std::lock_guard<std::mutex> lock(mutex_);
        return !asked_.empty();
    }
    // Waits up to `ms` for a build to finish.
    void wait(double ms) {
        std::unique_lock<std::mutex> lock(mutex_);
        finished_.wait_for(lock, std::chrono::duration<double, std::milli>(ms),
                           [this] { return !done_.empty(); });
    }

private:
    void work() {
        for (;;) {
            RegionKey k;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                wake_.wait(lock, [this] { return stopping_ || !jobs_.empty(); });
                if (stopping_) {
                    return;
                }
                k = jobs_.front();
                jobs_.pop_front();
            }
            Built b = build(k);
            {
                std::lock_guard<std::mutex> lock(mutex_);
                done_.push_back(std::move(b));
            }
            finished_.notify_all();
        }
    }

    Built build(const RegionKey& k) const {
        const auto t0 = std::chrono::steady_clock::now();
        Built b;
        b.key = k;
        const double spacing = std::ldexp(opt_.base_spacing, k.lod);
        const uint32_t cells = opt_.region_cells;
        const double side = spacing * cells;
        const double x0 = double(k.ix) * side, y0 = double(k.iy) * side;
        const tg_grid grid{cells, cells, x0, spacing, 0.0, y0 + side, 0.0, -spacing};
        std::vector<CraterRecord> recs(8192);
        std::vector<float> values(8192 * 24);
        std::vector<double> foot(8192 * 3);
        CraterShapeKernel kernel{};
        size_t nr = 0, nd = 0;
        for (int attempt = 0; attempt < 2; ++attempt) {
            b.status = tg_crater_batch(&opt_.craters, &opt_.shaping, &grid, &kernel, recs.data(),
                                       recs.size(), values.data(), values.size(), foot.data(),
                                       &nr, &nd);
            if (b.status != TG_OK || (nr <= recs.size() && nd <= values.size())) {
                break;
            }
            recs.resize(nr);
            values.resize(nd);
            foot.resize(3 * nr);
        }
        if (b.status == TG_OK) {
            // Owned records (centers in the region) first; an indexed region (the level point
            // queries read) keeps the others reaching in after them.
            const bool indexed = k.lod == pointLevel_;
            for (int pass = 0; pass < (indexed ? 2 : 1); ++pass) {
                for (size_t i = 0; i < nr; ++i) {
                    const double x = foot[3 * i], y = foot[3 * i + 1];
                    const bool owned = x >= x0 && x < x0 + side && y >= y0 && y < y0 + side;
                    if (owned != (pass == 0)) {
                        continue;
                    }
                    const CraterRecord& r = recs[i];
                    b.heavy |= r.tableCount > 0u || r.markCount > 0u || r.terraceCount > 0u ||
                               r.peakCount > 0u || r.shiftX != 0.0f || r.shiftY != 0.0f ||
                               r.upslopeX != 0.0f || r.upslopeY != 0.0f;
                    if (r.hasDatum == 1u) {
                        b.status = TG_ERROR_UNSUPPORTED;
                    }
                    b.records.push_back(r);
                    b.footprints.insert(b.footprints.end(),
                                        {foot[3 * i], foot[3 * i + 1], foot[3 * i + 2]});
                    b.culls.push_back(cull_of(r, values.data(), kernel.reachRadii));
                }
                if (pass == 0) {
                    b.owned = uint32_t(b.records.size());
                }
            }
            b.data.assign(values.begin(), values.begin() + std::ptrdiff_t(nd));
            if (indexed) {
                index(b, x0, y0, side);
            }
        }
        b.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                   .count();
        return b;
    }

    // Cell lists of an indexed region: each of kIndexCells^2 cells lists the records whose
    // footprint disk (the larger of reach and cull distance) meets it.
    static void index(Built& b, double x0, double y0, double side) {
        const uint32_t g = kIndexCells;
        const double cell = side / g;
        std::vector<std::vector<uint32_t>> cells(size_t(g) * g);
        for (uint32_t i = 0; i < b.records.size(); ++i) {
            const double x = b.footprints[3 * size_t(i)], y = b.footprints[3 * size_t(i) + 1];
            const double reach = std::fmax(b.footprints[3 * size_t(i) + 2], double(b.culls[i])) +
                                 1e-3;
            if (!std::isfinite(reach)) {
                for (auto& c : cells) {
                    c.push_back(i);
                }
                continue;
            }
            const int cx0 = std::max(0, int(std::floor((x - reach - x0) / cell)));
            const int cx1 = std::min(int(g) - 1, int(std::floor((x + reach - x0) / cell)));
            const int cy0 = std::max(0, int(std::floor((y - reach - y0) / cell)));
            const int cy1 = std::min(int(g) - 1, int(std::floor((y + reach - y0) / cell)));
            for (int cy = cy0; cy <= cy1; ++cy) {
                for (int cx = cx0; cx <= cx1; ++cx) {
                    const double bx0 = x0 + cx * cell, by0 = y0 + cy * cell;
                    const double dx = std::fmax(std::fmax(bx0 - x, x - (bx0 + cell)), 0.0);
                    const double dy = std::fmax(std::fmax(by0 - y, y - (by0 + cell)), 0.0);
                    if (dx * dx + dy * dy <= reach * reach) {
                        cells[size_t(cy) * g + size_t(cx)].push_back(i);
                    }
                }
            }
        }
        b.lists.assign(size_t(g) * g + 1, 0u);
        for (size_t c = 0; c < cells.size(); ++c) {
            b.lists[c + 1] = b.lists[c] + uint32_t(cells[c].size());
        }
        for (const auto& c : cells) {
            b.lists.insert(b.lists.end(), c.begin(), c.end());
        }
        b.index.x0 = x0;
        b.index.y0 = y0;
        b.index.cell = cell;
        b.index.g = g;
    }

    tg_server_options opt_{};
    int pointLevel_ = -1;
    std::vector<std::thread> threads_;
    std::mutex mutex_;
    std::condition_variable wake_, finished_;
    std::deque<RegionKey> jobs_;
    std::vector<Built> done_;
    std::unordered_set<RegionKey, RegionHash> asked_;
    bool stopping_ = false;
};

struct ServeSlot {
    tg_batch* batch = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t copied = nullptr;
    bool busy = false;
    std::vector<Pending> reqs;
    std::vector<uint64_t> offsets;  // output offset of each request
    std::vector<uint32_t> pitches;
    std::vector<RegionKey> used;
    Buffer out;
    float* host = nullptr;          // pinned mirror of the output
    size_t hostFloats = 0;
    size_t outFloats = 0;
    uint32_t replays = 0;           // the batch's graph launches when this one was enqueued
    uint64_t seq = 0;               // the server's launch count when it was launched
};

}  // namespace

struct tg_server {
    tg_device* dev = nullptr;
    tg_server_options opt{};
    BatchNoise noise{};
    std::vector<batch::Octave> octaves;
    CraterShapeKernel kernel{};
    bool fast = true;
    bool tuned = false;
    double margin = 0.0;  // meters a crater can reach beyond its region

    Buffer records, footprints, culls, data, harmonics, lists;
    uint32_t recCap = 0, dataCap = 0, listCap = 0;
    Ranges recRanges, dataRanges, listRanges;
    cudaStream_t installStream = nullptr;
    std::unordered_map<RegionKey, Region, RegionHash> regions;
    std::list<Pending> waiting;
    Builders builders;
    std::vector<Built> stash;  // built regions the arenas had no room for yet
    std::vector<ServeSlot> slots;
    uint64_t tick = 0;
    uint64_t launches = 0;
    tg_server_stats stats{};
};

namespace {

double level_spacing(const tg_server* s, int lod) {
    return std::ldexp(s->opt.base_spacing, lod);
}

// The level of detail of a spacing: base_spacing * 2^lod, or -1 when it is none.
int level_of(const tg_server* s, double spacing) {
    const double k = std::log2(spacing / s->opt.base_spacing);
    const double r = std::round(k);
    if (!(std::fabs(k - r) < 1e-9) || r < 0.0 || r > 30.0) {
        return -1;
    }
    return int(r);
}

size_t server_bytes(const tg_server* s) {
    size_t total = s->records.bytes + s->footprints.bytes + s->culls.bytes + s->data.bytes +
                   s->harmonics.bytes + s->lists.bytes;
    for (const ServeSlot& slot : s->slots) {
        total += slot.out.bytes + (slot.batch ? batch::device_bytes(slot.batch) : 0);
    }
    return total;
}

void note_bytes(tg_server* s) {
    s->stats.device_bytes = server_bytes(s);
    s->stats.peak_bytes = std::max(s->stats.peak_bytes, s->stats.device_bytes);
}

void evict(tg_server* s, std::unordered_map<RegionKey, Region, RegionHash>::iterator it) {
    s->recRanges.give(it->second.recBegin, it->second.recTotal);
    s->dataRanges.give(it->second.dataBegin, it->second.dataCount);
    s->listRanges.give(it->second.listBegin, it->second.listCount);
    s->regions.erase(it);
    ++s->stats.regions_evicted;
}

// Arena room for `records` records, `values` data floats and `entries` list words, evicting least
// recently used regions that no batch in flight reads.
bool make_room(tg_server* s, size_t records, size_t values, size_t entries, size_t& recAt,
               size_t& dataAt, size_t& listAt) {
    for (;;) {
        size_t r = 0, d = 0, l = 0;
        if (s->recRanges.take(records, r)) {
            if (s->dataRanges.take(values, d)) {
                if (s->listRanges.take(entries, l)) {
                    recAt = r;
                    dataAt = d;
                    listAt = l;
                    return true;
                }
                s->dataRanges.give(d, values);
            }
            s->recRanges.give(r, records);
        }
        auto victim = s->regions.end();
        for (auto it = s->regions.begin(); it != s->regions.end(); ++it) {
            if (it->second.inFlight == 0 &&
                (victim == s->regions.end() || it->second.lastUse < victim->second.lastUse)) {
                victim = it;
            }
        }
        if (victim == s->regions.end()) {
            return false;
        }
        evict(s, victim);
    }
}

// Copies built regions into the arenas (evicting least recently used idle regions); builds
// that find no room wait in the stash.
int install_regions(tg_server* s) {
    std::vector<Built> built = s->builders.take();
    for (Built& b : s->stash) {
        built.push_back(std::move(b));
    }
    s->stash.clear();
    for (Built& b : built) {
        if (b.status != TG_OK) {
            return fail(b.status, "building a feature region failed");
        }
        if (s->regions.count(b.key)) {
            continue;
        }
        size_t recAt = 0, dataAt = 0, listAt = 0;
        if (!make_room(s, b.records.size(), b.data.size(), b.lists.size(), recAt, dataAt,
                       listAt)) {
            s->stash.push_back(std::move(b));
            continue;
        }
        const cudaStream_t st = s->installStream;
        if (!b.records.empty()) {
            TG_CUDA(cudaMemcpyAsync(static_cast<CraterRecord*>(s->records.ptr) + recAt,
                                    b.records.data(), b.records.size() * sizeof(CraterRecord),
                                    cudaMemcpyHostToDevice, st),
                    "copy to device");
            TG_CUDA(cudaMemcpyAsync(static_cast<double*>(s->footprints.ptr) + 3 * recAt,
                                    b.footprints.data(), b.footprints.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, st),
                    "copy to device");
            TG_CUDA(cudaMemcpyAsync(static_cast<float*>(s->culls.ptr) + recAt, b.culls.data(),
                                    b.culls.size() * sizeof(float), cudaMemcpyHostToDevice, st),
                    "copy to device");
        }
        if (!b.data.empty()) {
            TG_CUDA(cudaMemcpyAsync(static_cast<float*>(s->data.ptr) + dataAt, b.data.data(),
                                    b.data.size() * sizeof(float), cudaMemcpyHostToDevice, st),
                    "copy to device");
        }
        if (!b.lists.empty()) {
            TG_CUDA(cudaMemcpyAsync(static_cast<uint32_t*>(s->lists.ptr) + listAt, b.lists.data(),
                                    b.lists.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                    st),
                    "copy to device");
        }
        // The lean path's harmonics of the region, once, where every batch reads them.
        TG_CUDA(launch_crater_harmonics(static_cast<const CraterRecord*>(s->records.ptr) + recAt,
                                        uint32_t(b.records.size()),
                                        static_cast<const float*>(s->data.ptr) + dataAt,
                                        static_cast<float*>(s->harmonics.ptr) + dataAt, st),
                "harmonics launch");
        TG_CUDA(cudaStreamSynchronize(st), "synchronize");
        if (b.heavy) {
            s->fast = false;
        }
        Region r;
        r.recBegin = uint32_t(recAt);
        r.recCount = b.owned;
        r.recTotal = uint32_t(b.records.size());
        r.dataBegin = uint32_t(dataAt);
        r.dataCount = uint32_t(b.data.size());
        r.listBegin = uint32_t(listAt);
        r.listCount = uint32_t(b.lists.size());
        r.index = b.index;
        r.index.recBase = uint32_t(recAt);
        r.index.dataBase = uint32_t(dataAt);
        r.index.listBase = uint32_t(listAt);
        r.lastUse = ++s->tick;
        s->regions.emplace(b.key, r);
        ++s->stats.regions_built;
        s->stats.region_ms += b.ms;
    }
    return TG_OK;
}

// The regions whose craters can reach the box (x0, y0, x1, y1) at level `lod`.
void keys_for(const tg_server* s, int lod, double x0, double y0, double x1, double y1,
              std::vector<RegionKey>& keys) {
    const double side = level_spacing(s, lod) * s->opt.region_cells;
    const int64_t ix0 = int64_t(std::floor((x0 - s->margin) / side));
    const int64_t ix1 = int64_t(std::floor((x1 + s->margin) / side));
    const int64_t iy0 = int64_t(std::floor((y0 - s->margin) / side));
    const int64_t iy1 = int64_t(std::floor((y1 + s->margin) / side));
    for (int64_t iy = iy0; iy <= iy1; ++iy) {
        for (int64_t ix = ix0; ix <= ix1; ++ix) {
            keys.push_back(RegionKey{lod, ix, iy});
        }
    }
}

// Whether every region a request needs is resident; asks the builders for the others.
bool ready(tg_server* s, const Pending& p) {
    bool all = true;
    for (const RegionKey& k : p.keys) {
        if (!s->regions.count(k)) {
            s->builders.request(k);
            all = false;
        }
    }
    return all;
}

// Enqueues on the slot's stream the copies of each request's heights: device requests straight
// into their buffers, host requests into the pinned mirror (copied out at completion). With
// `wait`, returns once they are done.
int deliver(ServeSlot& slot, bool wait) {
    for (size_t i = 0; i < slot.reqs.size(); ++i) {
        const tg_request& r = slot.reqs[i].req;
        const bool direct = r.memory == TG_MEMORY_DEVICE || slot.reqs[i].pinned;
        const float* src = static_cast<const float*>(slot.out.ptr) + slot.offsets[i];
        float* dst = direct ? r.heights : slot.host + slot.offsets[i];
        const cudaMemcpyKind kind =
            r.memory == TG_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (r.kind == 0 && direct) {
            TG_CUDA(cudaMemcpy2DAsync(dst, r.grid.width * sizeof(float), src,
                                      slot.pitches[i] * sizeof(float),
                                      r.grid.width * sizeof(float), r.grid.height, kind,
                                      slot.stream),
                    "copy out");
        } else {
            const size_t n = r.kind == 0 ? size_t(slot.pitches[i]) * r.grid.height : r.n_points;
            TG_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(float), kind, slot.stream), "copy out");
        }
    }
    if (wait) {
        TG_CUDA(cudaStreamSynchronize(slot.stream), "synchronize");
    }
    return TG_OK;
}

// Forms one batch from the waiting requests and launches it on `slot`.
int launch_slot(tg_server* s, ServeSlot& slot) {
    batch::Spec spec;
    spec.noise = s->noise;
    spec.octaves = s->octaves;
    spec.kernel = s->kernel;
    spec.features.records = static_cast<const CraterRecord*>(s->records.ptr);
    spec.features.footprints = static_cast<const double*>(s->footprints.ptr);
    spec.features.data = static_cast<const float*>(s->data.ptr);
    spec.features.harmonics = static_cast<float*>(s->harmonics.ptr);
    spec.features.harmonicsReady = true;  // computed when each region was installed
    spec.features.pointLists = static_cast<const uint32_t*>(s->lists.ptr);
    spec.features.culls = static_cast<const float*>(s->culls.ptr);
    std::unordered_map<RegionKey, uint32_t, RegionHash> table;  // region -> pointRegions index
    slot.reqs.clear();
    slot.offsets.clear();
    slot.pitches.clear();
    slot.used.clear();
    uint64_t cells = 0, outFloats = 0, bytes = 0;
    // Each slot's share of the budget left after the feature arenas bounds its batch.
    const uint64_t arenas = s->stats.feature_bytes;
    const uint64_t allowance =
        s->opt.hbm_budget > arenas ? (s->opt.hbm_budget - arenas) / s->slots.size() : 0;
    // Requests in arrival order whose regions are resident; the others wait for their builds.
    for (auto pit = s->waiting.begin(); pit != s->waiting.end();) {
        Pending& p = *pit;
        if (!ready(s, p)) {
            ++pit;
            continue;
        }
        if (!slot.reqs.empty() && cells + p.cells > s->opt.max_batch_cells) {
            break;
        }
        // Admission by memory: the request's output, bins and entries (about 6 B per cell) and
        // its (region, record) pairs (24 B each) within the slot's share of the budget; a batch
        // always takes its first request.
        uint64_t pairs = 0;
        for (const RegionKey& k : p.keys) {
            pairs += p.req.kind == 0 ? s->regions[k].recCount : 0u;
        }
        const uint64_t need = p.cells * 6 + pairs * 24;
        if (!slot.reqs.empty() && bytes + need > allowance) {
            ++s->stats.deferred;
            break;
        }
        bytes += need;
        const uint32_t item = uint32_t(spec.items.size());
        batch::Item it{};
        if (p.req.kind == 0) {
            const tg_grid& g = p.req.grid;
            to_grid(&g, it.grid);
            it.pitch = (g.width + 3u) & ~3u;
            it.points = false;
            it.pointBegin = 0xffffffffu;
            it.boulderWidth = 0.0;
            outFloats = (outFloats + 3u) & ~uint64_t(3);
            it.heightOffset = outFloats;
            outFloats += uint64_t(it.pitch) * g.height;
        } else {
            // Points read their regions' resident cell lists: no refs, no binning.
            const double side = level_spacing(s, p.lod) * s->opt.region_cells;
            it.grid = Grid{p.req.n_points, p.tw, double(p.ix0) * side, side, 0.0,
                           double(p.iy0) * side, 0.0, -side};
            it.pitch = p.th;
            it.points = true;
            it.kind = kTileIndexedPoints;
            it.pointBegin = uint32_t(spec.points.size() / 2);
            it.tableBase = uint32_t(spec.pointTable.size());
            it.boulderWidth = 0.0;
            it.dsSpacing = s->opt.point_spacing;
            it.heightOffset = outFloats;
            outFloats += p.req.n_points;
            spec.points.insert(spec.points.end(), p.xy.begin(), p.xy.end());
            for (uint32_t ry = 0; ry < p.th; ++ry) {
                for (uint32_t rx = 0; rx < p.tw; ++rx) {
                    uint32_t index = 0xffffffffu;
                    if (p.occupied[size_t(ry) * p.tw + rx]) {
                        const RegionKey k{p.lod, p.ix0 + rx, p.iy0 + ry};
                        auto found = table.find(k);
                        if (found == table.end()) {
                            found = table.emplace(k, uint32_t(spec.pointRegions.size())).first;
                            spec.pointRegions.push_back(s->regions[k].index);
                        }
                        index = found->second;
                    }
                    spec.pointTable.push_back(index);
                }
            }
        }
        for (const RegionKey& k : p.keys) {
            Region& r = s->regions[k];
            r.lastUse = ++s->tick;
            ++r.inFlight;  // held until the batch completes
            slot.used.push_back(k);
            if (p.req.kind == 0) {
                spec.refs.push_back(
                    BatchRef{item, r.recBegin, r.recCount, r.dataBegin, 0, 0, 0, 0});
            }
        }
        slot.offsets.push_back(it.heightOffset);
        slot.pitches.push_back(it.pitch);
        spec.items.push_back(it);
        cells += p.cells;
        slot.reqs.push_back(std::move(p));
        pit = s->waiting.erase(pit);
    }
    if (slot.reqs.empty()) {
        return TG_OK;
    }
    spec.fast = s->fast;
    if (s->opt.post_spacing > 0.0) {
        const tg_ds_options& r = s->opt.refine;
        spec.ds.on = true;
        spec.ds.postSpacing = s->opt.post_spacing;
        spec.ds.fractalDimension = r.fractal_dimension;
        spec.ds.scale = r.scale;
        spec.ds.minPixelSize = r.min_pixel_size;
        spec.ds.seed = r.seed;
        spec.ds.spline = r.interp == 1u;
    }
    if (int st = batch::load(slot.batch, std::move(spec))) {
        return st;
    }
    if (!s->tuned) {
        s->tuned = true;
        if (s->opt.variant >= 0) {
            if (int st = tg_batch_set_variant(slot.batch, s->opt.variant)) {
                return st;
            }
        } else if (int st = tg_batch_tune(slot.batch, 2, nullptr)) {
            return st;
        }
        tg_batch_stats bs{};
        tg_batch_stats_get(slot.batch, &bs);
        s->opt.variant = int(bs.variant);
        for (ServeSlot& o : s->slots) {
            if (&o != &slot && !o.busy) {
                if (int st = tg_batch_set_variant(o.batch, s->opt.variant)) {
                    return st;
                }
            }
        }
    }
    slot.outFloats = outFloats;
    TG_CUDA(slot.out.reserve(outFloats * sizeof(float)), "allocation");
    bool toHost = false;  // a pageable host request needs the pinned mirror
    for (const Pending& p : slot.reqs) {
        toHost |= p.req.memory == TG_MEMORY_HOST && !p.pinned;
    }
    if (toHost && slot.hostFloats < outFloats) {
        if (slot.host != nullptr) {
            cudaFreeHost(slot.host);
            slot.host = nullptr;
        }
        const size_t n = outFloats + outFloats / 2;
        TG_CUDA(cudaMallocHost(&slot.host, n * sizeof(float)), "pinned allocation");
        slot.hostFloats = n;
    }
    if (int st = batch::launch(slot.batch, static_cast<float*>(slot.out.ptr), slot.stream)) {
        return st;
    }
    slot.replays = batch::replays(slot.batch);
    slot.seq = ++s->launches;
    if (int st = deliver(slot, false)) {
        return st;
    }
    TG_CUDA(cudaEventRecord(slot.copied, slot.stream), "event record");
    slot.busy = true;
    ++s->stats.batches;
    note_bytes(s);
    return TG_OK;
}

// Hands back a finished slot's requests: heights copied into the callers' buffers.
int complete_slot(tg_server* s, ServeSlot& slot, uint64_t* ids, size_t capacity, size_t& count) {
    TG_CUDA(cudaEventSynchronize(slot.copied), "synchronize");
    if (int st = batch::finish(slot.batch)) {
        slot.busy = false;
        return st;
    }
    if (batch::replays(slot.batch) != slot.replays) {
        // The bins needed more entries and the batch ran again: deliver its heights once more.
        if (int st = deliver(slot, true)) {
            return st;
        }
    }
    tg_batch_stats bs{};
    tg_batch_stats_get(slot.batch, &bs);
    s->stats.gpu_ms += bs.graph_ms;
    for (size_t i = 0; i < slot.reqs.size(); ++i) {
        const Pending& p = slot.reqs[i];
        const float* src = slot.host + slot.offsets[i];
        if (p.req.memory == TG_MEMORY_DEVICE || p.pinned) {
            // Already copied by the slot's stream.
        } else if (p.req.kind == 0) {
            for (uint32_t r = 0; r < p.req.grid.height; ++r) {
                std::memcpy(p.req.heights + size_t(r) * p.req.grid.width,
                            src + size_t(r) * slot.pitches[i], p.req.grid.width * sizeof(float));
            }
        } else {
            std::memcpy(p.req.heights, src, p.req.n_points * sizeof(float));
        }
        if (count < capacity) {
            ids[count] = p.req.id;
        }
        ++count;
        ++s->stats.completed;
        s->stats.cells += p.cells;
    }
    for (const RegionKey& k : slot.used) {
        auto it = s->regions.find(k);
        if (it != s->regions.end() && it->second.inFlight > 0) {
            --it->second.inFlight;
        }
    }
    slot.reqs.clear();
    slot.used.clear();
    slot.busy = false;
    return TG_OK;
}

}  // namespace

extern "C" {

int tg_server_create(tg_device* device, const tg_server_options* options, tg_server** server) {
    if (server == nullptr || options == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "server and options are required");
    }
    *server = nullptr;
    if (int st = check_device(device)) {
        return st;
    }
    const tg_server_options& o = *options;
    if (!(o.base_spacing > 0.0) || !std::isfinite(o.base_spacing) || !(o.point_spacing > 0.0) ||
        o.slots < 1 || o.slots > 8 || o.region_cells < 16 || o.region_cells > 65536 ||
        o.max_batch_cells == 0 || o.hbm_budget == 0) {
        return fail(TG_ERROR_ARGUMENT, "server options out of range");
    }
    tg_server* s = new tg_server();
    s->dev = device;
    s->opt = o;
    auto undo = [&](int st) {
        tg_server_destroy(s);
        return st;
    };
    if (level_of(s, o.point_spacing) < 0) {
        return undo(fail(TG_ERROR_ARGUMENT, "point_spacing must be base_spacing * 2^k"));
    }
    if (o.post_spacing != 0.0 &&
        (!(o.post_spacing > 0.0) || !std::isfinite(o.post_spacing) ||
         !(o.refine.fractal_dimension >= 2.0 && o.refine.fractal_dimension <= 3.0) ||
         !(o.refine.scale >= 0.0) || !std::isfinite(o.refine.scale) ||
         !(o.refine.min_pixel_size >= 0.0) || o.refine.interp > 1u)) {
        return undo(fail(TG_ERROR_ARGUMENT, "refinement: post spacing > 0, fractal dimension in "
                                            "[2, 3], scale and min pixel size >= 0, interp 0 or 1"));
    }
    if (int st = batch::make_noise(o.fractals, o.n_fractals, o.elevation, s->noise,
                                   s->octaves)) {
        return undo(st);
    }
    // The crater kernel every region shares, from a one-cell batch.
    const tg_grid one{1, 1, 0.0, o.base_spacing, 0.0, o.base_spacing, 0.0, -o.base_spacing};
    size_t nr = 0, nd = 0;
    if (tg_crater_batch(&o.craters, &o.shaping, &one, &s->kernel, nullptr, 0, nullptr, 0, nullptr,
                        &nr, &nd) != TG_OK) {
        return undo(fail(TG_ERROR_ARGUMENT, "the crater population is invalid"));
    }
    s->fast = crater_fast_path(s->kernel, 0);
    // A crater's reach beyond its center: reachRadii x the largest outline stretch x radius.
    s->margin = double(s->kernel.reachRadii) * 2.5 * 0.5 * o.craters.max_diameter;
    // Feature arenas: a quarter of the budget, records and their footprints (168 B) and 24 data
    // floats per record.
    // Feature arenas: a quarter of the budget; per record its record, footprint and cull
    // (172 B), 24 data floats and their harmonics, and 4 list words.
    const size_t arenaBytes = size_t(o.hbm_budget / 4);
    const size_t perRecord = sizeof(CraterRecord) + 3 * sizeof(double) + sizeof(float) +
                             2 * 24 * sizeof(float) + 4 * sizeof(uint32_t);
    const size_t nRecords = std::max<size_t>(1024, std::min<size_t>(arenaBytes / perRecord,
                                                                    0x7fffffffu / 24));
    s->recCap = uint32_t(nRecords);
    s->dataCap = uint32_t(nRecords * 24);
    s->listCap = uint32_t(nRecords * 4);
    cudaError_t err = s->records.reserve(size_t(s->recCap) * sizeof(CraterRecord));
    if (err == cudaSuccess) {
        err = s->footprints.reserve(size_t(s->recCap) * 3 * sizeof(double));
    }
    if (err == cudaSuccess) {
        err = s->culls.reserve(size_t(s->recCap) * sizeof(float));
    }
    if (err == cudaSuccess) {
        err = s->data.reserve(size_t(s->dataCap) * sizeof(float));
    }
    if (err == cudaSuccess) {
        err = s->harmonics.reserve(size_t(s->dataCap) * sizeof(float));
    }
    if (err == cudaSuccess) {
        err = s->lists.reserve(size_t(s->listCap) * sizeof(uint32_t));
    }
    if (err == cudaSuccess) {
        err = cudaStreamCreateWithFlags(&s->installStream, cudaStreamNonBlocking);
    }
    if (err != cudaSuccess) {
        return undo(cuda_fail(err, "feature arena allocation"));
    }
    s->recRanges.reset(s->recCap);
    s->dataRanges.reset(s->dataCap);
    s->listRanges.reset(s->listCap);
    const unsigned cores = std::max(2u, std::thread::hardware_concurrency());
    s->builders.start(std::min(16u, cores - 1u), o, level_of(s, o.point_spacing));
    s->stats.feature_bytes = s->records.bytes + s->footprints.bytes + s->culls.bytes +
                             s->data.bytes + s->harmonics.bytes + s->lists.bytes;
    s->slots.resize(o.slots);
    for (ServeSlot& slot : s->slots) {
        if (int st = tg_batch_create(device, &slot.batch)) {
            return undo(st);
        }
        err = cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking);
        if (err == cudaSuccess) {
            err = cudaEventCreateWithFlags(&slot.copied, cudaEventDisableTiming);
        }
        if (err != cudaSuccess) {
            return undo(cuda_fail(err, "slot set-up"));
        }
    }
    note_bytes(s);
    *server = s;
    return TG_OK;
}

void tg_server_destroy(tg_server* s) {
    if (s == nullptr) {
        return;
    }
    if (s->dev != nullptr) {
        cudaSetDevice(s->dev->ordinal);
    }
    s->builders.stop();
    for (ServeSlot& slot : s->slots) {
        if (slot.stream != nullptr) {
            cudaStreamSynchronize(slot.stream);
        }
        if (slot.batch != nullptr) {
            batch::finish(slot.batch);
            tg_batch_destroy(slot.batch);
        }
        slot.out.release();
        if (slot.host != nullptr) {
            cudaFreeHost(slot.host);
        }
        if (slot.copied != nullptr) {
            cudaEventDestroy(slot.copied);
        }
        if (slot.stream != nullptr) {
            cudaStreamDestroy(slot.stream);
        }
    }
    s->records.release();
    s->footprints.release();
    s->culls.release();
    s->data.release();
    s->harmonics.release();
    s->lists.release();
    if (s->installStream != nullptr) {
        cudaStreamDestroy(s->installStream);
    }
    delete s;
}

int tg_server_submit(tg_server* s, const tg_request* request) {
    if (s == nullptr || request == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "server and request are required");
    }
    const tg_request& r = *request;
    Pending p;
    p.req = r;
    if (r.heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "request %llu: heights is null", (unsigned long long)r.id);
    }
    if (r.memory != TG_MEMORY_HOST && r.memory != TG_MEMORY_DEVICE) {
        return fail(TG_ERROR_ARGUMENT, "request %llu: memory is host or device",
                    (unsigned long long)r.id);
    }
    if (r.memory == TG_MEMORY_DEVICE && reinterpret_cast<uintptr_t>(r.heights) % 4u != 0u) {
        return fail(TG_ERROR_ARGUMENT, "request %llu: heights not 4-byte aligned",
                    (unsigned long long)r.id);
    }
    if (r.memory == TG_MEMORY_HOST) {
        // Page-locked host heights take the device-to-host copy directly; pageable ones go
        // through the slot's pinned mirror and a host copy at completion.
        cudaPointerAttributes a{};
        p.pinned = cudaPointerGetAttributes(&a, r.heights) == cudaSuccess &&
                   a.type == cudaMemoryTypeHost;
        (void)cudaGetLastError();
    }
    if (r.kind == 0) {
        Grid g;
        if (int st = to_grid(&r.grid, g)) {
            return st;
        }
        if (r.grid.pixel_width != -r.grid.pixel_height || r.grid.width == 0 ||
            r.grid.height == 0) {
            return fail(TG_ERROR_ARGUMENT, "request %llu: tiles have square pixels, north up",
                        (unsigned long long)r.id);
        }
        p.lod = level_of(s, r.grid.pixel_width);
        if (p.lod < 0) {
            return fail(TG_ERROR_ARGUMENT, "request %llu: spacing is not base_spacing * 2^k",
                        (unsigned long long)r.id);
        }
        p.cells = uint64_t(r.grid.width) * r.grid.height;
        keys_for(s, p.lod, r.grid.origin_x, r.grid.origin_y + r.grid.height * r.grid.pixel_height,
                 r.grid.origin_x + r.grid.width * r.grid.pixel_width, r.grid.origin_y, p.keys);
    } else if (r.kind == 1) {
        if (r.n_points == 0 || r.points == nullptr) {
            return fail(TG_ERROR_ARGUMENT, "request %llu: no points", (unsigned long long)r.id);
        }
        p.xy.assign(r.points, r.points + 2 * size_t(r.n_points));
        for (double v : p.xy) {
            if (!std::isfinite(v)) {
                return fail(TG_ERROR_ARGUMENT, "request %llu: a point is not finite",
                            (unsigned long long)r.id);
            }
        }
        p.lod = level_of(s, s->opt.point_spacing);
        p.cells = r.n_points;
        p.req.points = nullptr;
        // The regions holding the points (each lists every crater reaching into it), found in
        // a table over the regions of the points' bounding box.
        const double side = level_spacing(s, p.lod) * s->opt.region_cells;
        double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
        for (uint32_t i = 0; i < r.n_points; ++i) {
            lo[0] = std::min(lo[0], p.xy[2 * i]);
            lo[1] = std::min(lo[1], p.xy[2 * i + 1]);
            hi[0] = std::max(hi[0], p.xy[2 * i]);
            hi[1] = std::max(hi[1], p.xy[2 * i + 1]);
        }
        // Region (rx, ry) of the table as the device finds it: floor((x - x0) / side).
        p.ix0 = int64_t(std::floor(lo[0] / side));
        p.iy0 = int64_t(std::floor(lo[1] / side));
        const double ox = double(p.ix0) * side, oy = double(p.iy0) * side;
        const int64_t w = int64_t(std::floor((hi[0] - ox) / side)) + 1;
        const int64_t h = int64_t(std::floor((hi[1] - oy) / side)) + 1;
        if (w * h > (int64_t(1) << 22)) {
            return fail(TG_ERROR_UNSUPPORTED, "request %llu: points span too many regions",
                        (unsigned long long)r.id);
        }
        p.tw = uint32_t(w);
        p.th = uint32_t(h);
        p.occupied.assign(size_t(w * h), 0);
        for (uint32_t i = 0; i < r.n_points; ++i) {
            const int64_t rx = std::min(std::max<int64_t>(
                                            int64_t(std::floor((p.xy[2 * i] - ox) / side)), 0),
                                        w - 1);
            const int64_t ry = std::min(std::max<int64_t>(
                                            int64_t(std::floor((p.xy[2 * i + 1] - oy) / side)), 0),
                                        h - 1);
            p.occupied[size_t(ry * w + rx)] = 1;
        }
        for (int64_t ry = 0; ry < h; ++ry) {
            for (int64_t rx = 0; rx < w; ++rx) {
                if (p.occupied[size_t(ry * w + rx)]) {
                    p.keys.push_back(RegionKey{p.lod, p.ix0 + rx, p.iy0 + ry});
                }
            }
        }
    } else {
        return fail(TG_ERROR_ARGUMENT, "request kind is 0 (tile) or 1 (points)");
    }
    ready(s, p);  // start building its regions now
    s->waiting.push_back(std::move(p));
    ++s->stats.submitted;
    return TG_OK;
}

int tg_server_poll(tg_server* s, int wait, uint64_t* ids, size_t capacity, size_t* count) {
    if (s == nullptr || count == nullptr || (capacity > 0 && ids == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "server and count are required");
    }
    if (int st = check_device(s->dev)) {
        return st;
    }
    *count = 0;
    size_t n = 0;
    for (;;) {
        // Finished batches first (their slots free up), oldest first.
        for (ServeSlot& slot : s->slots) {
            if (slot.busy && cudaEventQuery(slot.copied) == cudaSuccess) {
                if (int st = complete_slot(s, slot, ids, capacity, n)) {
                    return st;
                }
            }
        }
        // Regions the builders finished, then the waiting requests into every free slot
        // (continuous batching).
        if (int st = install_regions(s)) {
            return st;
        }
        for (ServeSlot& slot : s->slots) {
            if (!slot.busy && !s->waiting.empty()) {
                if (int st = launch_slot(s, slot)) {
                    return st;
                }
            }
        }
        bool busy = false;
        for (const ServeSlot& slot : s->slots) {
            busy |= slot.busy;
        }
        if (!wait || n > 0 || (!busy && s->waiting.empty())) {
            break;
        }
        if (busy) {
            // Block on the batch launched first among those running.
            ServeSlot* oldest = nullptr;
            for (ServeSlot& slot : s->slots) {
                if (slot.busy && (oldest == nullptr || slot.seq < oldest->seq)) {
                    oldest = &slot;
                }
            }
            TG_CUDA(cudaEventSynchronize(oldest->copied), "synchronize");
        } else if (s->builders.busy()) {
            s->builders.wait(1.0);  // requests wait on their regions
        } else if (!s->stash.empty()) {
            return fail(TG_ERROR_MEMORY, "the feature arenas cannot hold the regions a request "
                                         "needs");
        }
    }
    *count = n;
    note_bytes(s);
    return TG_OK;
}

int tg_server_stats_get(tg_server* s, tg_server_stats* stats) {
    if (s == nullptr || stats == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "server and stats are required");
    }
    tg_server_stats out = s->stats;
    out.regions_resident = s->regions.size();
    out.device_bytes = server_bytes(s);
    *stats = out;
    return TG_OK;
}

}  // extern "C"
