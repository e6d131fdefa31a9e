// Host-side crater populations and kernel records on a plane: what a CraterLayer's ApplySamples
// hands the crater kernel, restated so the batched and served forms (and the benchmarks) can
// build their own batches without the reference library.
//
// The random draws must be the reference's bit for bit (the determinism contract,
// include/terraingen/pipeline/terrain.h:65-67), so the steps are kept in the reference's order:
//   Philox4x32-10 and RandomStream        (include/terraingen/random/philox.h:82, stream.cpp:7-27)
//   SamplePoisson (multiplication / PTRS) (src/random/samplers.cpp:14-55)
//   CraterBands, GenerateCellCraters,
//   the band plan and DrawKept filters    (src/layers/craters/generation/population.cpp)
//   CraterApplyOrder, ResolutionWeight    (apply_options.cpp:96, src/layers/fade.cpp:50)
//   FreshnessDegradation::State           (degradation/freshness_degradation.cpp)
//   IrregularOutline, power-law harmonics (shaping/irregularity.cpp:165-260)
//   BaseRecord / AppendKernelOutline      (shaping/crater_kernel.cpp:187, irregularity.cpp:295)
// This file is compiled with -ffp-contract=off and uses the host libm, as the reference does.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <unistd.h>

#include "../../include/tgb200.h"
#include "layouts.h"
#include "crater_records.h"
#include "population_plan.h"

namespace tgb {
namespace host {

// --- Philox4x32-10 and the keyed streams ----------------------------------------------------

struct Words4 {
    uint32_t x, y, z, w;
};

inline Words4 philox(Words4 c, uint32_t k0, uint32_t k1) {
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = uint64_t(0xD2511F53u) * c.x;
        const uint64_t p1 = uint64_t(0xCD9E8D57u) * c.z;
        c = Words4{uint32_t(p1 >> 32) ^ c.y ^ k0, uint32_t(p1), uint32_t(p0 >> 32) ^ c.w ^ k1,
                   uint32_t(p0)};
    }
    return c;
}

// Philox4x32-10 of n counters held as four word arrays, in place: the blocks of many streams at
// once, in a loop the host compiler vectorizes across counters (one build per vector width, the
// widest the host supports taken at load time). Integer work only, so every build gives the
// bits `philox` gives.
__attribute__((target_clones("avx512f", "avx2", "default"))) void philox_soa(
    uint32_t* __restrict x, uint32_t* __restrict y, uint32_t* __restrict z,
    uint32_t* __restrict w, size_t n, uint32_t k0, uint32_t k1) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t cx = x[i], cy = y[i], cz = z[i], cw = w[i];
        uint32_t a = k0, b = k1;
        for (int round = 0; round < 10; ++round) {
            if (round > 0) {
                a += 0x9E3779B9u;
                b += 0xBB67AE85u;
            }
            const uint64_t p0 = uint64_t(0xD2511F53u) * cx;
            const uint64_t p1 = uint64_t(0xCD9E8D57u) * cz;
            const uint32_t nx = uint32_t(p1 >> 32) ^ cy ^ a;
            const uint32_t nz = uint32_t(p0 >> 32) ^ cw ^ b;
            cy = uint32_t(p1);
            cw = uint32_t(p0);
            cx = nx;
            cz = nz;
        }
        x[i] = cx;
        y[i] = cy;
        z[i] = cz;
        w[i] = cw;
    }
}

// Stream tags (include/terraingen/random/streams.h:15-26).
constexpr uint32_t kCraterStream = 0x43524154u;
constexpr uint32_t kCraterAgeStream = 0x43524147u;
constexpr uint32_t kCraterIdStream = 0x43524944u;
constexpr uint32_t kCraterSlopeStream = 0x534C4F50u;
constexpr uint32_t kCraterTerraceStream = 0x54455252u;
constexpr uint32_t kCraterPeakStream = 0x5045414Bu;
constexpr uint32_t kCraterIrregularityStream = 0x49525247u;
constexpr uint32_t kCraterTextureStream = 0x54455854u;
constexpr uint32_t kCraterNoiseStream = 0x434E4F53u;
constexpr uint32_t kBoulderCandidateStream = 0x524F434Bu;  // streams.h:31
constexpr uint32_t kBoulderAttributeStream = 0x41545452u;  // streams.h:32

class Stream {
  public:
    Stream(uint32_t seed, uint32_t stream, uint32_t a = 0, uint32_t b = 0, uint32_t c = 0)
        : k0_(seed), k1_(stream), counter_{a, b, c, 0u} {}

    uint32_t next_u32() {
        if (used_ == 4) {
            block_ = philox(counter_, k0_, k1_);
            ++counter_.w;
            used_ = 0;
        }
        const uint32_t words[4] = {block_.x, block_.y, block_.z, block_.w};
        return words[used_++];
    }

    double next_double() {
        const uint64_t high = next_u32() >> 5u;
        const uint64_t low = next_u32() >> 6u;
        return double((high << 26u) | low) * 0x1p-53;
    }

  private:
    uint32_t k0_, k1_;
    Words4 counter_;
    Words4 block_{};
    int used_ = 4;
};

uint32_t substream_seed(uint32_t seed, uint32_t stream, uint32_t a = 0) {
    return philox(Words4{a, 0u, 0u, 0xFFFFFFFFu}, seed, stream).x;
}

uint32_t pcg(uint32_t v) {  // include/terraingen/noise/hash.h:33
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

uint32_t crater_key(uint64_t id, uint32_t seed) {  // crater.h:99, hash.h:68 HashWord64
    return pcg(uint32_t(id) ^ pcg(uint32_t(id >> 32u) ^ seed));
}

uint64_t poisson(Stream& random, double mean) {
    if (mean == 0.0) {
        return 0;
    }
    if (mean < 10.0) {
        const double limit = std::exp(-mean);
        uint64_t count = 0;
        double product = random.next_double();
        while (product > limit) {
            ++count;
            product *= random.next_double();
        }
        return count;
    }
    // Hoermann's transformed rejection with squeeze (PTRS).
    const double sqrtMean = std::sqrt(mean);
    const double logMean = std::log(mean);
    const double b = 0.931 + 2.53 * sqrtMean;
    const double a = -0.059 + 0.02483 * b;
    const double inverseAlpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    while (true) {
        const double u = random.next_double() - 0.5;
        const double v = random.next_double();
        const double us = 0.5 - std::fabs(u);
        const double k = std::floor((2.0 * a / us + b) * u + mean + 0.43);
        if (us >= 0.07 && v <= vr) {
            return uint64_t(k);
        }
        if (k < 0.0 || (us < 0.013 && v > us)) {
            continue;
        }
        if (std::log(v) + std::log(inverseAlpha) - std::log(a / (us * us) + b) <=
            -mean + k * logMean - std::lgamma(k + 1.0)) {
            return uint64_t(k);
        }
    }
}

// --- the population ---------------------------------------------------------------------------

struct Box {
    double minX, minY, maxX, maxY;
    Box expanded(double m) const { return Box{minX - m, minY - m, maxX + m, maxY + m}; }
    bool contains(double x, double y) const {
        return x >= minX && x < maxX && y >= minY && y < maxY;
    }
};

struct Crater {
    double x, y, diameter, age;
    uint64_t id;
};

struct Band {
    int exponent;
    double low, high, cellSize;
};

std::vector<Band> crater_bands(double minD, double maxD, double factor) {
    std::vector<Band> bands;
    for (int k = std::ilogb(minD); std::ldexp(1.0, k) < maxD; ++k) {
        const double low = std::fmax(minD, std::ldexp(1.0, k));
        const double high = std::fmin(maxD, std::ldexp(1.0, k + 1));
        bands.push_back({k, low, high, factor * std::ldexp(1.0, k + 1)});
    }
    return bands;
}

// N(>=D) = c D^-e (PowerLawSfd, include/terraingen/distribution/power_law.h:20-33). With
// `weight` > 0 it is instead the one-term SummedSfd `weight` x that law (summed.cpp:33-47), which
// a boulder layer draws its candidates from: the sum has no closed-form inverse, so a diameter is
// found as SizeFrequencyDistribution::InvertCumulative does (size_frequency.cpp:34-113), by
// Illinois steps on log N over log D, then bisection if they stall.
struct PowerLaw {
    double c, e;
    double weight = 0.0;

    double law(double d) const { return c * std::pow(d, -e); }
    double cumulative(double d) const { return weight > 0.0 ? 0.0 + weight * law(d) : law(d); }
    double incremental(double d) const {
        const double one = c * e * std::pow(d, -e - 1.0);
        return weight > 0.0 ? 0.0 + weight * one : one;
    }
    double expected(double lo, double hi) const { return 1.0 * (cumulative(lo) - cumulative(hi)); }
    double sample(Stream& random, double lo, double hi) const {
        return sample(random, lo, hi, expected(lo, hi), cumulative(lo));
    }
    // The same draw with the band's expected count and cumulative(lo) made once by the caller.
    double sample(Stream& random, double lo, double hi, double count, double top) const {
        const double target = top - random.next_double() * count;
        const double d = weight > 0.0 ? invert(target, lo, hi) : std::pow(target / c, -1.0 / e);
        return std::clamp(d, lo, hi);
    }

    // The diameter in [lo, hi] where N = target.
    double invert(double target, double lo, double hi) const {
        double low = std::log(lo), high = std::log(hi);
        if (target > 0.0) {
            const double logTarget = std::log(target);
            const auto excess = [&](double u) {
                return std::log(cumulative(std::exp(u))) - logTarget;
            };
            // Illinois regula falsi on the bracket [a, b] (util/numerics.h:33-61).
            double a = low, b = high, fa = excess(low), fb = excess(high);
            int side = 0;
            if (!(fa > 0.0)) {
                return std::exp(low);
            }
            if (!(fb < 0.0)) {
                return std::exp(high);
            }
            double u = low;
            bool stalled = true;
            for (int i = 0; i < 100; ++i) {
                const double previous = u;
                const double secant = b - fb * (b - a) / (fb - fa);
                u = secant > a && secant < b ? secant : 0.5 * (a + b);
                const double g = excess(u);
                if (std::isnan(g)) {
                    break;
                }
                if (g == 0.0 || std::fabs(u - previous) <= 1e-14 * std::fmax(1.0, std::fabs(u))) {
                    stalled = false;
                    break;
                }
                if ((g < 0.0) == (fa < 0.0)) {
                    a = u;
                    fa = g;
                    fb *= side == -1 ? 0.5 : 1.0;
                    side = -1;
                } else {
                    b = u;
                    fb = g;
                    fa *= side == 1 ? 0.5 : 1.0;
                    side = 1;
                }
            }
            if (!stalled) {
                return std::exp(u);
            }
            low = a;
            high = b;
        }
        const double tolerance = 1e-15 * std::fmax(1.0, std::fabs(high));
        for (int i = 0; i < 200 && high - low > tolerance; ++i) {
            const double middle = 0.5 * (low + high);
            (!(cumulative(std::exp(middle)) > target) ? high : low) = middle;
        }
        return std::exp(0.5 * (low + high));
    }
};

int32_t cell_coordinate(double v) {
    return int32_t(v);
}

// GenerateCellCraters on a plane (population.cpp:381): sink(crater) for each in draw order.
template <typename Sink>
void each_cell_crater(const Band& band, int32_t i, int32_t j, const PowerLaw& law,
                      double lifetime, uint32_t seed, const Sink& sink) {
    const uint32_t k = uint32_t(band.exponent);
    Stream geometry(seed, kCraterStream, uint32_t(i), uint32_t(j), k);
    Stream ages(seed, kCraterAgeStream, uint32_t(i), uint32_t(j), k);
    const double perArea = law.expected(band.low, band.high);
    const double top = law.cumulative(band.low);
    const double area = band.cellSize * band.cellSize;
    const uint64_t count = poisson(geometry, perArea * area);
    for (uint64_t index = 0; index < count; ++index) {
        const double diameter = law.sample(geometry, band.low, band.high, perArea, top);
        const double u = geometry.next_double();
        const double v = geometry.next_double();
        const double x = (i + u) * band.cellSize;
        const double y = (j + v) * band.cellSize;
        const double age = std::clamp(ages.next_double() * lifetime, 0.0, lifetime);
        const Words4 id = philox(Words4{uint32_t(i), uint32_t(j), k, uint32_t(index)}, seed,
                                 kCraterIdStream);
        sink(Crater{x, y, diameter, age, (uint64_t(id.x) << 32) | id.y});
    }
}

std::vector<Crater> cell_craters(const Band& band, int32_t i, int32_t j, const PowerLaw& law,
                                 double lifetime, uint32_t seed) {
    std::vector<Crater> out;
    each_cell_crater(band, i, j, law, lifetime, seed, [&](const Crater& c) { out.push_back(c); });
    return out;
}

// Host threads the batch builders use (tg_set_host_threads); 0 for every core.
std::atomic<unsigned> g_host_threads{0};

unsigned host_threads() {
    const unsigned asked = g_host_threads.load();
    const unsigned cores = std::max(1u, std::thread::hardware_concurrency());
    return std::min(asked == 0 ? cores : asked, 256u);
}

// Runs body(i) for every i in [0, n) on up to `threads` host threads, the caller's included;
// items are taken in order from a shared counter, so each runs exactly once.
// Host worker threads kept for the life of the process: a call hands them its loop instead of
// starting threads of its own (tens of microseconds each, several loops a batch). One call at a
// time holds them; a call made while another holds them (the served form's region builders run
// batches side by side), or in a process forked after they started, runs on threads of its own.
class HostPool {
  public:
    static HostPool& instance() {
        static HostPool* pool = new HostPool();  // never destroyed: its threads wait until exit
        return *pool;
    }

    // body(i) for every i < n on `workers` threads, the caller one of them; false, with nothing
    // run, when the pool is held or belongs to the process this one was forked from.
    template <typename Body>
    bool run(size_t n, size_t workers, const Body& body) {
        std::unique_lock<std::mutex> held(m_held, std::try_to_lock);
        if (!held.owns_lock() || getpid() != m_pid) {
            return false;
        }
        std::unique_lock<std::mutex> lock(m_mutex);
        while (m_started < workers - 1) {
            std::thread(&HostPool::serve, this, m_started++).detach();
        }
        m_call = [](const void* context, size_t i) { (*static_cast<const Body*>(context))(i); };
        m_context = &body;
        m_n = n;
        m_next.store(0);
        m_want = workers - 1;
        m_finished = 0;
        ++m_generation;
        lock.unlock();
        m_wake.notify_all();
        drain();
        lock.lock();
        m_done.wait(lock, [&] { return m_finished == m_want; });
        return true;
    }

  private:
    HostPool() : m_pid(getpid()) {}

    void drain() {
        for (size_t i = m_next.fetch_add(1); i < m_n; i = m_next.fetch_add(1)) {
            m_call(m_context, i);
        }
    }

    // A worker: each generation it is one of the m_want first, it drains the loop and reports.
    void serve(size_t id) {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lock(m_mutex);
        for (;;) {
            m_wake.wait(lock, [&] { return m_generation != seen; });
            seen = m_generation;
            if (id >= m_want) {
                continue;
            }
            lock.unlock();
            drain();
            lock.lock();
            if (++m_finished == m_want) {
                m_done.notify_one();
            }
        }
    }

    const pid_t m_pid;
    std::mutex m_held, m_mutex;
    std::condition_variable m_wake, m_done;
    size_t m_started = 0, m_want = 0, m_finished = 0, m_n = 0;
    uint64_t m_generation = 0;
    std::atomic<size_t> m_next{0};
    void (*m_call)(const void*, size_t) = nullptr;
    const void* m_context = nullptr;
};

template <typename Body>
void parallel_for(size_t n, unsigned threads, const Body& body) {
    const size_t workers = std::min<size_t>(threads, n);
    if (workers <= 1) {
        for (size_t i = 0; i < n; ++i) {
            body(i);
        }
        return;
    }
    if (HostPool::instance().run(n, workers, body)) {
        return;
    }
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
            body(i);
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(workers - 1);
    for (size_t t = 1; t < workers; ++t) {
        pool.emplace_back(work);
    }
    work();
    for (std::thread& t : pool) {
        t.join();
    }
}

// Craters over `region` with their candidate margin (GenerateCraters, planar, no spacing,
// density map or manual craters), into `out`, those for which `wanted` holds. Each band's row of
// generation cells is drawn on its own (by `threads` host threads when asked), and the rows are
// joined in the reference's order: bands ascending, rows j, cells i, craters in draw order. The
// rows' lists are kept per calling thread from call to call, so repeated calls allocate nothing
// once they have grown.
template <typename Wanted>
void generate_into(const tg_crater_population& spec, const Box& region, const PowerLaw& law,
                   unsigned threads, const Wanted& wanted, std::vector<Crater>& result) {
    const double marginRadii = spec.margin_radii;
    auto margin = [&](double d) { return 0.5 * marginRadii * d; };
    struct Row {
        Band band;
        int32_t j, iMin, iMax;
        Box inner, outer;
    };
    std::vector<Row> rows;
    for (const Band& band : crater_bands(spec.min_diameter, spec.max_diameter,
                                         spec.cell_size_factor)) {
        if (band.high <= spec.min_resolved_diameter) {
            continue;
        }
        const Box cover = region.expanded(margin(band.high));
        const int32_t iMin = cell_coordinate(std::floor(cover.minX / band.cellSize));
        const int32_t jMin = cell_coordinate(std::floor(cover.minY / band.cellSize));
        const int32_t iMax = cell_coordinate(std::ceil(cover.maxX / band.cellSize) - 1.0);
        const int32_t jMax = cell_coordinate(std::ceil(cover.maxY / band.cellSize) - 1.0);
        for (int32_t j = jMin; j <= jMax; ++j) {
            rows.push_back(Row{band, j, iMin, iMax, region.expanded(margin(band.low)),
                               region.expanded(margin(band.high))});
        }
    }
    // The calling thread's lists, named by reference: inside the loop body, run on other
    // threads, the thread_local's own name would be theirs.
    static thread_local std::vector<std::vector<Crater>> keptRows;
    std::vector<std::vector<Crater>>& drawn = keptRows;
    if (drawn.size() < rows.size()) {
        drawn.resize(rows.size());
    }
    parallel_for(rows.size(), threads, [&](size_t q) {
        const Row& row = rows[q];
        const Band& band = row.band;
        const int32_t j = row.j;
        const Box& inner = row.inner;
        const Box& outer = row.outer;
        std::vector<Crater>& out = drawn[q];
        out.clear();
        for (int32_t i = row.iMin; i <= row.iMax; ++i) {
            // CellCraters::Rows(outer y range): the draw order, filtered by y.
            each_cell_crater(band, i, j, law, spec.lifetime_gyr, spec.seed, [&](const Crater& c) {
                if (!(c.y >= outer.minY && c.y <= outer.maxY)) {
                    return;
                }
                const bool inBand = c.diameter >= band.low && c.diameter <= band.high;
                if (inBand && !outer.contains(c.x, c.y)) {
                    return;
                }
                bool keep;
                if (!inBand) {
                    keep = region.expanded(margin(c.diameter)).contains(c.x, c.y);
                } else {
                    keep = inner.contains(c.x, c.y) ||
                           region.expanded(margin(c.diameter)).contains(c.x, c.y);
                }
                if (keep && wanted(c)) {
                    out.push_back(c);
                }
            });
        }
    });
    // Rows joined in order: each row's craters copied to its offset on the host threads.
    std::vector<size_t> base(rows.size() + 1, 0);
    for (size_t q = 0; q < rows.size(); ++q) {
        base[q + 1] = base[q] + drawn[q].size();
    }
    result.resize(base.back());
    parallel_for(rows.size(), threads, [&](size_t q) {
        std::copy(drawn[q].begin(), drawn[q].end(), result.begin() + base[q]);
    });
}

std::vector<Crater> generate(const tg_crater_population& spec, const Box& region,
                             const PowerLaw& law, unsigned threads = 1) {
    std::vector<Crater> out;
    generate_into(spec, region, law, threads, [](const Crater&) { return true; }, out);
    return out;
}

// The plan the device generator follows: per band, its cells, SamplePoisson's and
// PowerLawSfd::Sample's constants and the keep boxes, as `generate` uses them.
std::vector<CraterBandPlan> crater_plan(const tg_crater_population& spec, const double* r) {
    const Box region{r[0], r[1], r[2], r[3]};
    const PowerLaw law{spec.sfd_coefficient, spec.sfd_exponent};
    const double marginRadii = spec.margin_radii;
    auto margin = [&](double d) { return 0.5 * marginRadii * d; };
    std::vector<CraterBandPlan> plan;
    uint64_t cells = 0;
    for (const Band& band : crater_bands(spec.min_diameter, spec.max_diameter,
                                         spec.cell_size_factor)) {
        if (band.high <= spec.min_resolved_diameter) {
            continue;
        }
        CraterBandPlan p{};
        p.exponent = uint32_t(band.exponent);
        p.low = band.low;
        p.high = band.high;
        p.cellSize = band.cellSize;
        const Box cover = region.expanded(margin(band.high));
        p.iMin = cell_coordinate(std::floor(cover.minX / band.cellSize));
        p.jMin = cell_coordinate(std::floor(cover.minY / band.cellSize));
        p.iMax = cell_coordinate(std::ceil(cover.maxX / band.cellSize) - 1.0);
        p.jMax = cell_coordinate(std::ceil(cover.maxY / band.cellSize) - 1.0);
        p.mean = law.expected(band.low, band.high) * (band.cellSize * band.cellSize);
        p.limit = std::exp(-p.mean);
        p.sqrtMean = std::sqrt(p.mean);
        p.logMean = std::log(p.mean);
        p.b = 0.931 + 2.53 * p.sqrtMean;
        p.a = -0.059 + 0.02483 * p.b;
        p.inverseAlpha = 1.1239 + 1.1328 / (p.b - 3.4);
        p.vr = 0.9277 - 3.6224 / (p.b - 2.0);
        p.logInverseAlpha = std::log(p.inverseAlpha);
        p.count = law.expected(band.low, band.high);
        p.top = law.cumulative(band.low);
        p.inverseExponent = -1.0 / law.e;
        const Box inner = region.expanded(margin(band.low));
        const Box outer = region.expanded(margin(band.high));
        const double in[4] = {inner.minX, inner.minY, inner.maxX, inner.maxY};
        const double out[4] = {outer.minX, outer.minY, outer.maxX, outer.maxY};
        std::copy(in, in + 4, p.inner);
        std::copy(out, out + 4, p.outer);
        p.firstCell = cells;
        if (p.iMax >= p.iMin && p.jMax >= p.jMin) {
            cells += uint64_t(p.iMax - p.iMin + 1) * uint64_t(p.jMax - p.jMin + 1);
        }
        plan.push_back(p);
    }
    return plan;
}

void cell_kept(const tg_crater_population& spec, const double* r, const CraterBandPlan& p,
               int32_t i, int32_t j, std::vector<HostCrater>& out) {
    const Box region{r[0], r[1], r[2], r[3]};
    const PowerLaw law{spec.sfd_coefficient, spec.sfd_exponent};
    auto margin = [&](double d) { return 0.5 * spec.margin_radii * d; };
    const Band band{int(p.exponent), p.low, p.high, p.cellSize};
    const Box inner{p.inner[0], p.inner[1], p.inner[2], p.inner[3]};
    const Box outer{p.outer[0], p.outer[1], p.outer[2], p.outer[3]};
    for (const Crater& c : cell_craters(band, i, j, law, spec.lifetime_gyr, spec.seed)) {
        if (!(c.y >= outer.minY && c.y <= outer.maxY)) {
            continue;
        }
        const bool inBand = c.diameter >= band.low && c.diameter <= band.high;
        if (inBand && !outer.contains(c.x, c.y)) {
            continue;
        }
        const bool keep = inBand ? inner.contains(c.x, c.y) ||
                                       region.expanded(margin(c.diameter)).contains(c.x, c.y)
                                 : region.expanded(margin(c.diameter)).contains(c.x, c.y);
        if (keep) {
            out.push_back(HostCrater{c.x, c.y, c.diameter, c.age, c.id});
        }
    }
}

// --- preparation and records ----------------------------------------------------------------

double smoothstep(double t) {
    t = std::clamp(t, 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}

double resolution_weight(double diameter, double spacing, double start = 2.0,
                         double end = 4.0) {
    // 1 - Falloff(D / spacing, start, end, Smoothstep) (src/layers/fade.cpp:18-52)
    const double x = diameter / spacing;
    double f;
    if (x <= start) {
        f = 1.0;
    } else if (x >= end) {
        f = 0.0;
    } else {
        f = 1.0 - smoothstep((x - start) / (end - start));
    }
    return 1.0 - f;
}

struct Outline {
    double ellipticity = 1.0, heading = 0.0;
    double amplitudes[11], phases[11];  // the first `harmonics` of them
    int harmonics = 0;
    int firstHarmonic = 2;
};

// IrregularOutline with the default irregularity (power-law harmonics 2-12, roughness uniform
// in [0.01, 0.03], slope 1.5, 5.4% elliptical with ellipticity uniform in [1.1, 1.5]).
// The default outline's per-harmonic power law, k^-slope for k = 2..12, and sqrt(2 / sum of
// k^-2 slope): the same host pow calls for every crater, made once.
struct OutlineLaw {
    double power[11];
    double scale;
    OutlineLaw() {
        const double slope = 1.5;
        double sum = 0.0;
        for (int k = 2; k <= 12; ++k) {
            sum += std::pow(double(k), -2.0 * slope);
        }
        scale = std::sqrt(2.0 / sum);
        for (int k = 2; k <= 12; ++k) {
            power[k - 2] = std::pow(double(k), -slope);
        }
    }
};

// The words IrregularOutline draws, at most kOutlineDraws doubles: blocks 0 to 9 of the crater's
// irregularity stream (counter id low, id high, 0, block), as Stream would hand them out.
constexpr int kOutlineDraws = 20;
constexpr int kOutlineBlocks = kOutlineDraws / 2;

// The outline words of `n` craters (ids[i]) at once, words[i * 4 kOutlineBlocks + 4 b + lane].
void outline_words(const uint64_t* ids, size_t n, uint32_t seed, std::vector<uint32_t>& words) {
    const size_t lanes = n * kOutlineBlocks;
    static thread_local std::vector<uint32_t> soa;
    soa.resize(4 * lanes);
    uint32_t *x = soa.data(), *y = x + lanes, *z = y + lanes, *w = z + lanes;
    for (size_t i = 0; i < n; ++i) {
        for (int b = 0; b < kOutlineBlocks; ++b) {
            const size_t q = i * kOutlineBlocks + b;
            x[q] = uint32_t(ids[i]);
            y[q] = uint32_t(ids[i] >> 32);
            z[q] = 0u;
            w[q] = uint32_t(b);
        }
    }
    philox_soa(x, y, z, w, lanes, seed, kCraterIrregularityStream);
    words.resize(4 * lanes);
    for (size_t q = 0; q < lanes; ++q) {
        words[4 * q] = x[q];
        words[4 * q + 1] = y[q];
        words[4 * q + 2] = z[q];
        words[4 * q + 3] = w[q];
    }
}

// Stream::next_double from two consecutive words.
inline double unit_double(const uint32_t* words) {
    const uint64_t high = words[0] >> 5u;
    const uint64_t low = words[1] >> 6u;
    return double((high << 26u) | low) * 0x1p-53;
}

// IrregularOutline from the crater's outline words (outline_words).
Outline irregular_outline(const uint32_t* words) {
    static const OutlineLaw law;
    Outline o;
    struct {
        const uint32_t* at;
        double next_double() {
            const double v = unit_double(at);
            at += 2;
            return v;
        }
    } random{words};
    double d[9];
    for (double& v : d) {
        v = random.next_double();
    }
    const double rough = d[0], elongated = d[1], r1 = d[2], s1 = d[4], e1 = d[6], h = d[8];
    (void)s1;
    if (elongated < 0.054) {
        o.ellipticity = 1.1 + (1.5 - 1.1) * e1;  // clamped to (-inf, inf)
        o.heading = 3.14159265358979323846 * h;
    }
    if (rough < 1.0) {
        const double roughness = 0.01 + (0.03 - 0.01) * r1;  // clamped to (-inf, inf)
        const double norm = roughness * law.scale;
        o.firstHarmonic = 2;
        if (roughness > 0.0) {
            for (int k = 2; k <= 12; ++k) {
                o.amplitudes[o.harmonics] = norm * law.power[k - 2];
                o.phases[o.harmonics] = 2.0 * 3.14159265358979323846 * random.next_double();
                ++o.harmonics;
            }
        }
    }
    return o;
}

// Whether the footprint box of half-width `reach` around (x, y) holds a cell of the grid:
// Surface::Expand, then MappedBounds of GeoTransform::WorldToPixel over the box's corners
// (src/raster/cell_loops.cpp:21-28, geo_transform.h:70), then ClampIndex.
bool footprint_cells(const tg_grid& grid, double x, double y, double reach) {
    const double det = grid.pixel_width * grid.pixel_height - grid.row_rotation * grid.col_rotation;
    double minX = INFINITY, minY = INFINITY, maxX = -INFINITY, maxY = -INFINITY;
    if (grid.row_rotation == 0.0 && grid.col_rotation == 0.0 && grid.pixel_width > 0.0 &&
        grid.pixel_height < 0.0 && reach >= 0.0) {
        // Unrotated and north-up: det < 0, the column coordinate rises with x and the row
        // coordinate falls with y (rounding keeps both monotone), so two corners give the box's
        // extremes, by the same expressions.
        const auto px = [&](double wx, double wy) {
            return ((wx - grid.origin_x) * grid.pixel_height -
                    (wy - grid.origin_y) * grid.row_rotation) / det;
        };
        const auto py = [&](double wx, double wy) {
            return ((wy - grid.origin_y) * grid.pixel_width -
                    (wx - grid.origin_x) * grid.col_rotation) / det;
        };
        minX = px(x - reach, y - reach);
        maxX = px(x + reach, y - reach);
        minY = py(x - reach, y + reach);
        maxY = py(x - reach, y - reach);
    } else {
        for (const double wx : {x - reach, x + reach}) {
            for (const double wy : {y - reach, y + reach}) {
                const double dx = wx - grid.origin_x;
                const double dy = wy - grid.origin_y;
                const double px = (dx * grid.pixel_height - dy * grid.row_rotation) / det;
                const double py = (dy * grid.pixel_width - dx * grid.col_rotation) / det;
                minX = std::fmin(minX, px);
                minY = std::fmin(minY, py);
                maxX = std::fmax(maxX, px);
                maxY = std::fmax(maxY, py);
            }
        }
    }
    const double w = grid.width, h = grid.height;
    const double c0 = std::clamp(std::floor(minX), 0.0, w);
    const double c1 = std::clamp(std::ceil(maxX), 0.0, w);
    const double r0 = std::clamp(std::floor(minY), 0.0, h);
    const double r1 = std::clamp(std::ceil(maxY), 0.0, h);
    return size_t(c0) < size_t(c1) && size_t(r0) < size_t(r1);
}

double max_outline_scale(bool irregular) {  // MaxOutlineScale (irregularity.cpp:279)
    if (!irregular) {
        return 1.0;
    }
    const double rough = 1.0 + 0.03 * std::sqrt(2.0 * 11);
    return rough * std::sqrt(1.5);
}

// --- profile heights ------------------------------------------------------------------------
//
// The reference's CraterProfile::Height implementations evaluate the kernel header's float math
// (fassett_thomson.cpp:14, martin_parkes_dunstan.cpp, complex.cpp:70-78, on
// include/terraingen/layers/kernels/craters.h:330-505). Terrace records sample them, so they are
// restated here in float, in the header's operation order (this unit is compiled with
// -ffp-contract=off and calls the host libm's powf and sqrtf, as the reference's build does).

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kDegree = kPi / 180.0;
constexpr float kKernelPiF = 3.14159265358979f;

// The shape fields of a record (KernelStateRecord, profiles/profile.h:34).
struct ShapeState {
    float diameter, freshDepth, freshRim, currentDepth, currentRim;
};

ShapeState shape_state(double diameter, double freshDepth, double freshRim, double currentDepth,
                       double currentRim) {
    return ShapeState{float(diameter), float(freshDepth), float(freshRim), float(currentDepth),
                      float(currentRim)};
}

float ft_exterior(float x, float start) {  // craters.h:330
    const float polynomial =
        0.188253307f + x * (-0.187050452f + x * (0.01844746f + x * 0.01505647f));
    const float u = (x - start) / (1.5f - start);
    return polynomial * (1.0f - u * u);
}

float ft_shape(float x, uint32_t rim, float freshRim, float currentDepth) {  // craters.h:337
    if (x > 1.5f) {
        return 0.0f;
    }
    const float interior =
        -0.228809953f + x * (0.227533882f + x * (0.083116795f - x * 0.039499407f));
    float h = 0.0f;
    if (rim == 2u) {
        h = x <= 0.98f ? interior : (x <= 1.02f ? freshRim : ft_exterior(x, 1.02f));
    } else {
        const float edge = rim == 0u ? 0.98f : 1.0f;
        h = x <= 0.2f ? -0.181f : (x <= edge ? interior : ft_exterior(x, edge));
    }
    return std::max(h, freshRim - currentDepth);
}

struct ProfilePoint {
    float height, slope;
};

ProfilePoint mpd_exterior(float x, float rim, float ejectaScale) {  // craters.h:377
    const float offset = rim - ejectaScale;
    const float gradient = -ejectaScale / 8.0f - offset;
    const float r = 1.0f / (x + 1.0f);
    const float law = ejectaScale * r * r * r + offset + gradient * x;
    const float lawSlope = -3.0f * ejectaScale * r * r * r * r + gradient;
    const float taper = 1.0f - x * x;
    return ProfilePoint{law * taper, lawSlope * taper - 2.0f * x * law};
}

float mpd_height(float distance, float diameter, const ShapeState& c) {  // craters.h:391
    const float depth = c.currentDepth * diameter;
    const float rim = c.currentRim * diameter;
    const float freshRim = c.freshRim * diameter;
    const float radius = 0.5f * diameter;
    const float x = distance / radius - 1.0f;
    if (x >= 1.0f) {
        return 0.0f;
    }
    const float k = freshRim - rim + depth;
    const float alpha = (rim - freshRim) / k;
    if (x <= alpha) {
        return (k * x + 2.0f * k) * x + freshRim;
    }
    if (x <= 0.0f) {
        return k * (alpha + 1.0f) / alpha * x * x + rim;
    }
    const float scale = 0.14f * std::pow(radius, 0.74f);  // KernelEjectaScale
    const float ejectaScale = freshRim > 0.0f ? scale * rim / freshRim : scale;
    const float beta = std::min(1.0f, 1.5f * (freshRim - rim) / k);
    if (x <= beta) {
        const ProfilePoint join = mpd_exterior(beta, rim, ejectaScale);
        const float drop = rim - join.height;
        const float slope = drop > 0.0f ? std::max(join.slope, -3.0f * drop / beta) : join.slope;
        const float t = x / beta;
        return rim + (join.height - rim) * t * t * (3.0f - 2.0f * t) +
               beta * slope * t * t * (t - 1.0f);
    }
    return mpd_exterior(x, rim, ejectaScale).height;
}

float kilometer_law(float coefficient, float exponent, float diameter, bool volume) {
    const float kilometers = coefficient * std::pow(diameter / 1000.0f, exponent);
    return volume ? kilometers * 1e9f : kilometers * 1000.0f;
}

// The lunar complex shape (LunarComplexCraterShape) from a transition diameter, in the kernel's
// form (SetKernelComplexShape, complex.cpp:37-52).
void set_complex_shape(CraterProfileKernel& p, double transition) {
    p.complex = 1u;
    p.transitionDiameter = float(transition);
    p.floorCoefficient = float(0.187);
    p.floorExponent = float(1.249);
    p.peakHeightCoefficient = float(0.589e-3);
    p.peakHeightExponent = float(1.969);
    p.peakWidthCoefficient = float(0.987e-7);  // the peak volume law: no peak diameter law
    p.peakWidthExponent = float(5.078);
    p.peakFromVolume = 1u;
    p.peakFitMaxDiameter = float(51000.0);
    p.ejectaExponent = 3.0f;
    p.complexReachRadii = 3.0f;
}

float complex_height(const CraterProfileKernel& p, float distance, float diameter,
                     const ShapeState& c) {  // ComplexProfileHeight, craters.h:477
    const float radius = 0.5f * diameter;
    const float x = distance / radius;
    const float depth = c.currentDepth * diameter;
    const float rim = c.currentRim * diameter;
    if (x >= 1.0f) {
        if (x >= p.complexReachRadii) {
            return 0.0f;
        }
        const float edge = std::pow(p.complexReachRadii, -p.ejectaExponent);
        return rim * (std::pow(x, -p.ejectaExponent) - edge) / (1.0f - edge);
    }
    const float floorShare = std::min(
        0.9f, kilometer_law(p.floorCoefficient, p.floorExponent, diameter, false) / diameter);
    float height = rim - depth;
    if (x > floorShare) {
        const float t = (x - floorShare) / (1.0f - floorShare);
        height += depth * t * t;
    }
    // KernelComplexPeak and KernelPeakDome (craters.h:446-471), lowered by the kept depth.
    const float fitted =
        p.peakFitMaxDiameter > 0.0f ? std::min(diameter, p.peakFitMaxDiameter) : diameter;
    float peakHeight = kilometer_law(p.peakHeightCoefficient, p.peakHeightExponent, fitted, false);
    float base;
    if (p.peakFromVolume == 1u) {
        const float volume = kilometer_law(p.peakWidthCoefficient, p.peakWidthExponent, fitted, true);
        base = std::sqrt(3.0f * volume / (kKernelPiF * peakHeight));
    } else {
        base = 0.5f * kilometer_law(p.peakWidthCoefficient, p.peakWidthExponent, fitted, false);
    }
    base *= diameter / fitted;
    float dome = 0.0f;
    if (distance < base) {
        const float u = 1.0f - (distance / base) * (distance / base);
        dome = peakHeight * u * u;
    }
    const float kept = c.freshDepth > 0.0f ? c.currentDepth / c.freshDepth : 1.0f;
    return height + kept * dome;
}

// The layer's profile as CraterProfile::Height evaluates it (in double, from float math).
struct LayerProfile {
    uint32_t simple = 0;  // 0 Fassett-Thomson (Original rim), 1 Martin-Parkes-Dunstan
    bool complex = false;
    double transition = 0.0;
    CraterProfileKernel kernel{};  // the complex profile's own kernel form

    double simple_reach() const { return simple == 1u ? 2.0 : 1.5; }
    // ComplexCraterProfile::ReachRadii (complex.cpp:66): the larger of the two reaches.
    double reach() const { return complex ? std::fmax(simple_reach(), 3.0) : simple_reach(); }
    bool is_complex(double diameter) const { return complex && diameter >= transition; }

    double height(double distance, double diameter, const ShapeState& s) const {
        if (is_complex(diameter)) {
            return double(complex_height(kernel, float(distance), float(diameter), s));
        }
        const float d = float(diameter);
        if (simple == 1u) {
            return double(mpd_height(float(distance), d, s));
        }
        return double(ft_shape(float(distance) / (0.5f * d), 0u, s.freshRim, s.currentDepth) * d);
    }
};

// --- wall terraces (AppendKernelTerraces, crater_kernel.cpp:312-509) --------------------------

struct TerraceOptions {  // CraterTerraces' defaults (apply_options.h:183-226)
    double onset = 20000.0, full = 65000.0;
    int minBenches = 1, maxBenches = 4;
    double benchSlopeDegrees = 3.0, scarpShare = 0.25, scarpSlopeDegrees = 35.0;
    double arcShare = 0.6, rimVariation = 0.08, blockOffset = 0.6, blockGaps = 0.25;
    double minFreshness = 0.3;
};

float terrace_ease(float v, float rounding) {  // KernelTerraceEase, craters.h:968
    const float steepest = 1.0f / (1.0f - 0.5f * rounding);
    if (v < rounding) {
        return steepest * v * v / (2.0f * rounding);
    }
    return steepest * (v - 0.5f * rounding);
}

// The record's terraces, appended to `data`: the constants of the reference's terrace
// construction (bench arcs, step bases by wall height, scarp scallops and block offsets, bench
// levels that keep each step's mean height) and its draws, in its order.
void append_terraces(const TerraceOptions& t, uint32_t seed, const LayerProfile& profile,
                     double diameter, uint64_t id, double freshDepth, double freshRim,
                     double currentDepth, double currentRim, CraterRecord& record,
                     std::vector<float>& data) {
    constexpr double kFullCover = 0.9, kArcWidth = 0.3, kNarrowest = 0.25, kRounding = 0.4;
    constexpr double kMostScarp = 0.9, kSteepStep = 0.7, kSqueeze = 0.75, kScarpRoom = 0.4;
    constexpr double kScarpReach = 1.2, kMinScallops = 6.0, kMaxScallops = 12.0;
    constexpr double kRimScallop = 0.5, kLevelMargin = 0.1;
    constexpr int kWallSamples = 256, kMeanSamples = 64, kLevelIterations = 30;
    if (diameter < t.onset) {
        return;
    }
    const ShapeState s = shape_state(diameter, freshDepth, freshRim, currentDepth, currentRim);
    const double freshness = freshDepth > 0.0 ? currentDepth / freshDepth : 1.0;
    const double strength = smoothstep((freshness - t.minFreshness) / (1.0 - t.minFreshness));
    if (!(strength > 0.0)) {
        return;
    }
    // The floor edge: the lunar shape's floor law, which is also the default (Pike's).
    const double floorAt = double(kilometer_law(float(0.187), float(1.249), float(diameter), false));
    const double inner = std::clamp(floorAt / diameter, 0.2, 0.9);
    const double radius = 0.5 * diameter;
    const double drop =
        profile.height(radius, diameter, s) - profile.height(inner * radius, diameter, s);
    const double meanSlope = drop / ((1.0 - inner) * radius);
    const double benchSlope = std::tan(t.benchSlopeDegrees * kDegree);
    const double scarpSlope =
        std::tan(t.scarpSlopeDegrees * kDegree) * (1.0 - 0.5 * kRounding) * kSqueeze;
    const double slopeShare =
        meanSlope > 0.0 ? std::clamp(benchSlope / meanSlope, 0.02, 0.5) : 0.5;
    const double size = std::clamp((diameter - t.onset) / (t.full - t.onset), 0.0, 1.0);
    Stream random(seed, kCraterTerraceStream, uint32_t(id), uint32_t(id >> 32));
    const double spread = t.maxBenches - t.minBenches;
    const int benches = std::clamp(
        int(std::lround(t.minBenches + spread * size + random.next_double() - 0.5)),
        t.minBenches, t.maxBenches);
    // Bench arcs: harmonics 2..6 with weights 1/k normalised, random phases.
    double arcs[10];
    {
        double total = 0.0;
        for (int k = 2; k < 7; ++k) {
            total += 1.0 / k;
        }
        for (int k = 2; k < 7; ++k) {
            arcs[2 * (k - 2)] = 1.0 / k / total;
            arcs[2 * (k - 2) + 1] = 2.0 * kPi * random.next_double();
        }
    }
    const double cover =
        t.arcShare >= 1.0 ? 1.0 : t.arcShare + std::max(0.0, kFullCover - t.arcShare) * size;
    double cut = -2.0;
    if (cover < 1.0) {
        constexpr size_t kSamples = 360;
        std::vector<double> values(kSamples);
        for (size_t n = 0; n < kSamples; ++n) {
            const double theta = 2.0 * kPi * double(n) / double{kSamples};
            double sum = 0.0;
            for (size_t k = 0; k < 5; ++k) {
                sum += arcs[2 * k] * std::cos((double(k) + 2.0) * theta + arcs[2 * k + 1]);
            }
            values[n] = sum;
        }
        const auto at = values.begin() + std::ptrdiff_t((1.0 - cover) * double{kSamples - 1});
        std::nth_element(values.begin(), at, values.end());
        cut = *at;
    }
    record.terraceCount = uint32_t(benches);
    record.terraceOffset = uint32_t(data.size());
    for (const double v : {inner, slopeShare, strength, kRounding, cut, kArcWidth}) {
        data.push_back(float(v));
    }
    for (const double v : arcs) {
        data.push_back(float(v));
    }
    auto scallopCount = [&random] {
        return kMinScallops + std::floor((kMaxScallops - kMinScallops + 1.0) * random.next_double());
    };
    const double rimScallop =
        kRimScallop * t.rimVariation * strength * (0.6 + 0.8 * random.next_double());
    {
        // Drawn left to right, as the reference's braced list is.
        const double count = scallopCount();
        const double phase = random.next_double();
        for (const double v : {rimScallop, count, phase, t.blockGaps}) {
            data.push_back(float(v));
        }
    }
    // The wall's running-maximum height from the floor edge to the rim, 257 samples.
    std::vector<double> wall(kWallSamples + 1);
    for (size_t n = 0; n < wall.size(); ++n) {
        const double u = double(n) / kWallSamples;
        const double h = profile.height((inner + u * (1.0 - inner)) * radius, diameter, s);
        wall[n] = n == 0 ? h : std::max(h, wall[n - 1]);
    }
    const double rise = wall.back() - wall.front();
    auto across = [&](double share) {
        if (!(rise > 0.0)) {
            return share;
        }
        const double target = wall.front() + share * rise;
        const auto above = std::lower_bound(wall.begin(), wall.end(), target);
        if (above == wall.begin()) {
            return 0.0;
        }
        if (above == wall.end()) {
            return 1.0;
        }
        const double n = double(above - wall.begin());
        const double gap = *above - *(above - 1);
        const double part = gap > 0.0 ? (*above - target) / gap : 0.0;
        return (n - part) / kWallSamples;
    };
    std::vector<double> heights{0.0};
    double total = 0.0;
    for (int i = 0; i < benches; ++i) {
        total += 0.5 + random.next_double();
        heights.push_back(total);
    }
    std::vector<double> bases;
    for (double& h : heights) {
        h /= total;
        bases.push_back(across(h));
    }
    bases.back() = 1.0;
    const double narrowest = kNarrowest / benches;
    for (size_t k = 1; k + 1 < bases.size(); ++k) {
        bases[k] = std::max(bases[k], bases[k - 1] + narrowest);
    }
    for (size_t k = bases.size() - 2; k > 0; --k) {
        bases[k] = std::min(bases[k], bases[k + 1] - narrowest);
    }
    const double variation = t.rimVariation / (1.0 - inner);
    for (size_t k = 1; k < bases.size() - 1; ++k) {
        const double room = kScarpRoom * std::min(bases[k] - bases[k - 1], bases[k + 1] - bases[k]);
        double scallop = std::min(variation * (0.6 + 0.8 * random.next_double()), 0.9 * room);
        const double scallops = scallopCount();
        const double phase = random.next_double();
        double wobble = std::min(0.5 * variation * random.next_double(), 0.4 * room);
        const double wobblePhase = 2.0 * kPi * random.next_double();
        double block = t.blockOffset * room;
        const double reach = 2.0 / 3.0 * scallop + wobble + block;
        if (reach > kScarpReach * room) {
            const double fit = kScarpReach * room / reach;
            scallop *= fit;
            wobble *= fit;
            block *= fit;
        }
        const double key = double(random.next_u32() >> 8u);
        for (const double v : {bases[k], scallop, scallops, phase, wobble, wobblePhase, block, key}) {
            data.push_back(float(v));
        }
    }
    auto wallAt = [&](double u) {
        const double at = std::clamp(u, 0.0, 1.0) * kWallSamples;
        const size_t n = std::min(size_t(at), wall.size() - 2);
        return wall[n] + (at - double(n)) * (wall[n + 1] - wall[n]);
    };
    auto stairAt = [&](double within, double level, double scarp) {
        const float rounding = float(kRounding);
        const double lower = scarp * level;
        const double upper = scarp * (1.0 - level);
        double stair = level;
        if (within < lower) {
            stair = level * (1.0 - double{terrace_ease(float(1.0 - within / lower), rounding)});
        } else if (within > 1.0 - upper) {
            stair = level + (1.0 - level) *
                                double{terrace_ease(float((within - (1.0 - upper)) / upper),
                                                    rounding)};
        }
        return slopeShare * within + (1.0 - slopeShare) * stair;
    };
    auto meanHeight = [&](double from, double to, double level, double scarp) {
        double weighted = 0.0, weights = 0.0;
        for (int n = 0; n < kMeanSamples; ++n) {
            const double within = (n + 0.5) / kMeanSamples;
            const double r = inner + (from + within * (to - from)) * (1.0 - inner);
            const double shaped = level < 0.0 ? within : stairAt(within, level, scarp);
            weighted += r * wallAt(from + shaped * (to - from));
            weights += r;
        }
        return weighted / weights;
    };
    for (size_t k = 0; k + 1 < bases.size(); ++k) {
        const double from = bases[k], to = bases[k + 1];
        const double stepSlope = (wallAt(to) - wallAt(from)) / ((to - from) * (1.0 - inner) * radius);
        const double needed =
            scarpSlope > benchSlope ? (stepSlope - benchSlope) / (scarpSlope - benchSlope) : 1.0;
        const double scarp = std::clamp(needed, t.scarpShare, kMostScarp);
        const double kept = 1.0 - smoothstep((needed - kSteepStep) / (1.0 - kSteepStep));
        const double target = meanHeight(from, to, -1.0, scarp);
        // Bisect (util/numerics.h:23) for the level whose stair keeps the mean height.
        double low = kLevelMargin, high = 1.0 - kLevelMargin;
        for (int i = 0; i < kLevelIterations && high - low > 0.0; ++i) {
            const double middle = 0.5 * (low + high);
            (!(meanHeight(from, to, middle, scarp) < target) ? high : low) = middle;
        }
        for (const double v : {0.5 * (low + high), scarp, kept}) {
            data.push_back(float(v));
        }
    }
}

// --- central peaks (AppendKernelPeaks, crater_kernel.cpp:524-579) ----------------------------

struct PeakOptions {  // CraterPeaks' defaults (apply_options.h:241-268)
    int minMassifs = 1, maxMassifs = 4;
    double spreadRadii = 0.8, elongation = 2.0, chainSpreadDegrees = 70.0, sharpness = 0.6;
    double lopsidedness = 0.5, heightVariation = 0.5, roughness = 0.35;
    double roughnessWavelength = 0.35, warp = 0.12, heightScale = 1.0, widthScale = 1.0;
};

void append_peaks(const PeakOptions& o, uint32_t seed, uint64_t id, double freshDepth,
                  double currentDepth, CraterRecord& record, std::vector<float>& data) {
    constexpr double kPeakRoom = 2.3, kMainRadius = 1.0, kLesserRadius = 0.6, kMaxPull = 0.45;
    const double freshness =
        freshDepth > 0.0 ? std::clamp(currentDepth / freshDepth, 0.0, 1.0) : 1.0;
    Stream random(seed, kCraterPeakStream, uint32_t(id), uint32_t(id >> 32));
    const int massifs =
        o.minMassifs + std::min(o.maxMassifs - o.minMassifs,
                                int((o.maxMassifs - o.minMassifs + 1) * random.next_double()));
    record.peakCount = uint32_t(massifs);
    record.peakOffset = uint32_t(data.size());
    const double key = double(random.next_u32() >> 8u);
    for (const double v : {o.roughness * freshness, o.roughnessWavelength, o.warp, key,
                           o.heightScale, o.widthScale}) {
        data.push_back(float(v));
    }
    const double chain = 2.0 * kPi * random.next_double();
    const double room = kPeakRoom - o.warp;
    for (int n = 0; n < massifs; ++n) {
        // One draw per line below except where a main massif takes a constant, in this order.
        const bool main = n == 0;
        const double side = n % 2 == 0 ? kPi : 0.0;
        const double bearing =
            main ? 2.0 * kPi * random.next_double()
                 : chain + side + o.chainSpreadDegrees * kDegree * (random.next_double() - 0.5);
        const double reach =
            o.spreadRadii * (main ? 0.25 * random.next_double() : 0.35 + 0.65 * random.next_double());
        const double aspect = 1.0 + (o.elongation - 1.0) * random.next_double();
        const double stretch = std::sqrt(aspect);
        const double crowding = massifs == 1 ? 1.0 : std::sqrt(2.0 / massifs);
        double radius =
            crowding * (main ? kMainRadius : kLesserRadius * (0.5 + random.next_double()));
        radius = std::max(0.1, std::min(radius, (room - reach) / stretch));
        const double heading =
            main ? 2.0 * kPi * random.next_double() : bearing + 0.5 * (random.next_double() - 0.5);
        const double height = main ? 1.0 : 1.0 - o.heightVariation * random.next_double();
        const double exponent = std::clamp(
            (2.0 - 1.5 * o.sharpness) * (0.8 + 0.4 * random.next_double()), 0.4, 2.5);
        const double pull = kMaxPull * o.lopsidedness * std::sqrt(random.next_double());
        const double pullBearing = 2.0 * kPi * random.next_double();
        for (const double v : {reach * std::cos(bearing), reach * std::sin(bearing), radius, stretch,
                               std::cos(heading), std::sin(heading), height, exponent,
                               pull * std::cos(pullBearing), pull * std::sin(pullBearing),
                               2.0 - o.sharpness}) {
            data.push_back(float(v));
        }
    }
}

// The records of a block of consecutive craters in apply order, with data offsets relative to
// the block's own data until the blocks are placed in the outputs.
struct RecordBlock {
    std::vector<CraterRecord> records;
    std::vector<float> values;
    std::vector<double> foot;
};

// A batch builder's working arrays, kept per calling thread so that repeated batches reuse
// their memory: the drawn craters, the apply order's buckets and the record blocks.
struct BatchWork {
    std::vector<Crater> craters;
    std::vector<uint32_t> bucket, sorted, moved, slots;
    std::vector<RecordBlock> blocks;
};

// A batch's settings from the caller's population, shaping and grid: the layer profile, the
// terrace and peak options, the spacing, the grid's bounds and the population with the layer's
// candidate margins.
struct BatchSetup {
    LayerProfile profile;
    TerraceOptions terraces;
    PeakOptions peaks;
    double spacing = 0.0;
    Box bounds{};
    tg_crater_population p{};
    bool irregular = false;
    double reachRadii = 0.0;
};

int batch_setup(const tg_crater_population& spec, const tg_crater_shaping& shaping,
                const tg_grid& grid, BatchSetup& out) {
    if (grid.row_rotation != 0.0 || grid.col_rotation != 0.0 || !(grid.pixel_width > 0.0) ||
        !(grid.pixel_height < 0.0)) {
        return TG_ERROR_UNSUPPORTED;
    }
    if (shaping.profile > 3u) {
        return TG_ERROR_ARGUMENT;
    }
    LayerProfile& profile = out.profile;
    profile.simple = shaping.profile & 1u;
    profile.complex = shaping.profile >= 2u;
    if (profile.complex) {
        // ValidateComplexCraterShape (complex.cpp:19): a positive transition diameter.
        if (!(shaping.transition_diameter > 0.0) || !std::isfinite(shaping.transition_diameter)) {
            return TG_ERROR_ARGUMENT;
        }
        profile.transition = shaping.transition_diameter;
        set_complex_shape(profile.kernel, profile.transition);
    }
    TerraceOptions& terraces = out.terraces;
    if (shaping.terrace_onset > 0.0) {
        // ValidateCraterTerraces (apply_options.cpp:20): full above onset, min freshness in [0, 1).
        if (!(shaping.terrace_full > shaping.terrace_onset) ||
            !(shaping.terrace_min_freshness >= 0.0 && shaping.terrace_min_freshness < 1.0)) {
            return TG_ERROR_ARGUMENT;
        }
        terraces.onset = shaping.terrace_onset;
        terraces.full = shaping.terrace_full;
        terraces.minFreshness = shaping.terrace_min_freshness;
    }
    const double spacing = out.spacing = std::max(grid.pixel_width, -grid.pixel_height);
    // The grid's bounds (its cell edges), the region CraterLayer::ApplySamples draws over.
    out.bounds = Box{grid.origin_x, grid.origin_y + grid.height * grid.pixel_height,
                     grid.origin_x + grid.width * grid.pixel_width, grid.origin_y};
    tg_crater_population& p = out.p;
    p = spec;
    // DefaultCraterApply: irregular outlines, terraces and peaks; plain options: none.
    const bool irregular = out.irregular = shaping.irregular != 0;
    const double reachRadii = out.reachRadii = profile.reach();  // FT 1.5 R, MPD 2 R, complex 3 R
    p.margin_radii = reachRadii * max_outline_scale(irregular);
    p.min_resolved_diameter = std::fmax(2.0 * spacing, 0.0);
    return TG_OK;
}

// The batch's craters in apply order: the population drawn over the grid's bounds, the
// candidates kept as they are drawn, the order by the ages' buckets (work.craters and, in apply
// order, their indices work.sorted).
int batch_order(const BatchSetup& setup, const tg_grid& grid, unsigned threads, BatchWork& work,
                bool order = true) {
    // The craters that can give a record: a resolution weight above 0 and a footprint, grown
    // to the largest outline scale any crater can draw (MaxOutlineScale, irregularity.cpp:
    // 279, the bound the reference's own binning takes), that holds a cell of the grid. The
    // rest (most of the candidates the margins bring in) are dropped as they are drawn,
    // neither ordered nor built; the records are unchanged, as every crater left out would
    // be dropped by its exact footprint below, and the draw order of those kept stays theirs.
    const double growth = max_outline_scale(setup.irregular) * (1.0 + 1e-9);
    const tg_crater_population& p = setup.p;
    const double spacing = setup.spacing, reachRadii = setup.reachRadii;
    std::vector<Crater>& craters = work.craters;
    generate_into(p, setup.bounds, PowerLaw{p.sfd_coefficient, p.sfd_exponent}, threads,
                  [&](const Crater& c) {
                      return resolution_weight(c.diameter, spacing) != 0.0 &&
                             footprint_cells(grid, c.x, c.y,
                                             growth * reachRadii * (0.5 * c.diameter));
                  },
                  craters);
    if (craters.size() >= (size_t(1) << 32)) {
        return TG_ERROR_UNSUPPORTED;
    }
    if (!order) {
        return TG_OK;
    }
    const size_t nKept = craters.size();
    // The ages' range, by parts of 4096 craters on the host threads.
    constexpr size_t kPart = 4096;
    const size_t parts = (nKept + kPart - 1) / kPart;
    std::vector<double> partOldest(parts, -INFINITY), partYoungest(parts, INFINITY);
    parallel_for(parts, threads, [&](size_t part) {
        const size_t end = std::min(nKept, (part + 1) * kPart);
        double oldest = -INFINITY, youngest = INFINITY;
        for (size_t i = part * kPart; i < end; ++i) {
            oldest = std::fmax(oldest, craters[i].age);
            youngest = std::fmin(youngest, craters[i].age);
        }
        partOldest[part] = oldest;
        partYoungest[part] = youngest;
    });
    double oldest = -INFINITY, youngest = INFINITY;
    for (size_t part = 0; part < parts; ++part) {
        oldest = std::fmax(oldest, partOldest[part]);
        youngest = std::fmin(youngest, partYoungest[part]);
    }
    // CraterApplyOrder, oldest first (apply_options.cpp:96): age descending, then diameter
    // descending, id, draw index. The craters are spread over one bucket each on average by
    // age (floor((oldest - age) * scale): monotone in the age, so every bucket precedes the
    // next in the order and equal ages share one), put in bucket order by a stable radix
    // sort (two digits; per part counts, so each part writes its own slots and no thread
    // waits on another), then each run of one bucket is sorted by the whole comparison on
    // the host threads. The order is total, so it is the one the comparison defines,
    // whatever the ages' spread.
    const size_t buckets = std::max<size_t>(nKept, 1);
    const double spread = oldest - youngest;
    const double scale = spread > 0.0 ? double(buckets) / spread : 0.0;
    std::vector<uint32_t>& bucket = work.bucket;
    std::vector<uint32_t>& sorted = work.sorted;
    std::vector<uint32_t>& moved = work.moved;
    bucket.resize(nKept);
    sorted.resize(nKept);
    moved.resize(nKept);
    parallel_for(parts, threads, [&](size_t part) {
        const size_t end = std::min(nKept, (part + 1) * kPart);
        for (size_t i = part * kPart; i < end; ++i) {
            const double at = std::floor((oldest - craters[i].age) * scale);
            bucket[i] = uint32_t(std::clamp(at, 0.0, double(buckets - 1)));
            sorted[i] = uint32_t(i);
        }
    });
    int bits = 1;
    while (bits < 32 && (size_t(1) << bits) < buckets) {
        ++bits;
    }
    const int digitBits = (bits + 1) / 2;
    const size_t radix = size_t(1) << digitBits;
    std::vector<uint32_t>& slots = work.slots;
    slots.resize(parts * radix);
    for (int pass = 0; pass < 2; ++pass) {
        const int shift = pass * digitBits;
        const std::vector<uint32_t>& from = pass == 0 ? sorted : moved;
        std::vector<uint32_t>& to = pass == 0 ? moved : sorted;
        parallel_for(parts, threads, [&](size_t part) {
            uint32_t* count = slots.data() + part * radix;
            std::fill(count, count + radix, 0u);
            const size_t end = std::min(nKept, (part + 1) * kPart);
            for (size_t q = part * kPart; q < end; ++q) {
                ++count[(bucket[from[q]] >> shift) & (radix - 1)];
            }
        });
        uint32_t running = 0;
        for (size_t d = 0; d < radix; ++d) {
            for (size_t part = 0; part < parts; ++part) {
                const uint32_t n = slots[part * radix + d];
                slots[part * radix + d] = running;
                running += n;
            }
        }
        parallel_for(parts, threads, [&](size_t part) {
            uint32_t* slot = slots.data() + part * radix;
            const size_t end = std::min(nKept, (part + 1) * kPart);
            for (size_t q = part * kPart; q < end; ++q) {
                to[slot[(bucket[from[q]] >> shift) & (radix - 1)]++] = from[q];
            }
        });
    }
    const auto earlier = [&](uint32_t a, uint32_t b) {
        const Crater &ca = craters[a], &cb = craters[b];
        if (ca.age != cb.age) {
            return ca.age > cb.age;
        }
        if (ca.diameter != cb.diameter) {
            return ca.diameter > cb.diameter;
        }
        return ca.id != cb.id ? ca.id < cb.id : a < b;
    };
    // Runs of one bucket, sorted by the segment of kPart positions each run starts in.
    const auto same = [&](size_t q) { return bucket[sorted[q]] == bucket[sorted[q - 1]]; };
    parallel_for(parts, threads, [&](size_t part) {
        size_t q = part * kPart;
        const size_t limit = std::min(nKept, (part + 1) * kPart);
        while (q > 0 && q < limit && same(q)) {
            ++q;  // this run started in an earlier segment
        }
        while (q < limit) {
            size_t end = q + 1;
            while (end < nKept && same(end)) {
                ++end;
            }
            if (end - q > 1) {
                std::sort(sorted.begin() + q, sorted.begin() + end, earlier);
            }
            q = end;
        }
    });
    return TG_OK;
}

// The batch's CraterShapeKernel bytes into `kernel`.
void batch_shape_kernel(const BatchSetup& setup, void* kernel) {
    // MakeCraterShapeKernel (crater_kernel.cpp:277) for a simple FT or MPD profile and the
    // default shaping options.
    CraterShapeKernel k{};
    k.profile.ejectaExponent = 3.0f;
    k.profile.complexReachRadii = 3.0f;
    if (setup.profile.complex) {
        set_complex_shape(k.profile, setup.profile.transition);
    }
    k.profile.simple = setup.profile.simple == 1u ? kProfileMartinParkesDunstan
                                                  : kProfileFassettThomson;
    k.profile.tableExtent = 1.5f;
    k.reachRadii = float(setup.reachRadii);
    k.profileReachRadii = float(setup.reachRadii);
    k.blendStart = 0.8f;
    k.blendEnd = 1.2f;
    k.blendShape = 2u;
    k.replaceStart = 1.0f;
    k.replaceEnd = float(setup.reachRadii);
    k.ejectaReachRadii = 3.0f;
    k.rimInner = 0.8f;
    k.rimOuter = 1.2f;
    k.rimStrength = 1.0f;
    k.rimShape = 2u;
    k.noiseWavelength = 0.5f;
    k.noiseOctaves = 4;
    k.noiseGain = 0.5f;
    k.noiseRimWavelength = 0.1f;
    k.noiseRimInner = 0.8f;
    k.noiseRimOuter = 1.2f;
    k.wallStreakWidth = 0.15f;
    k.ejectaLineation = 0.15f;
    k.minFreshness = 0.5f;
    std::memcpy(kernel, &k, sizeof(k));
}

int record_plan(const tg_crater_population& spec, const tg_crater_shaping& shaping,
                const tg_grid& grid, void* kernel, RecordConstants& k,
                const std::function<RecordCrater*(size_t)>& place, size_t& count,
                std::vector<float>& extras) {
    BatchSetup setup;
    if (int st = batch_setup(spec, shaping, grid, setup)) {
        return st;
    }
    const unsigned threads = host_threads();
    static thread_local BatchWork workspace;
    BatchWork& work = workspace;
    if (int st = batch_order(setup, grid, threads, work, false)) {
        return st;
    }
    if (kernel != nullptr) {
        batch_shape_kernel(setup, kernel);
    }
    static const OutlineLaw law;
    k = RecordConstants{};
    k.originX = grid.origin_x;
    k.originY = grid.origin_y;
    k.pixelWidth = grid.pixel_width;
    k.pixelHeight = grid.pixel_height;
    k.rowRotation = grid.row_rotation;
    k.colRotation = grid.col_rotation;
    k.width = grid.width;
    k.height = grid.height;
    k.spacing = setup.spacing;
    k.reachRadii = setup.reachRadii;
    k.freshDepth = spec.depth_ratio;
    k.freshRim = spec.rim_ratio;
    for (int i = 0; i < 11; ++i) {
        k.outlinePower[i] = law.power[i];
    }
    k.outlineScale = law.scale;
    k.irregular = setup.irregular ? 1u : 0u;
    // SeededCraterApply (apply_options.cpp:57): every per-crater stream follows the layer seed.
    k.irregularitySeed = substream_seed(spec.seed, kCraterIrregularityStream);
    k.noiseSeed = substream_seed(spec.seed, kCraterNoiseStream);
    k.textureKeySeed = substream_seed(substream_seed(spec.seed, kCraterTextureStream),
                                      kCraterTextureStream);
    const uint32_t terraceSeed = substream_seed(spec.seed, kCraterTerraceStream);
    const uint32_t peakSeed = substream_seed(spec.seed, kCraterPeakStream);
    const double freshDepth = spec.depth_ratio, freshRim = spec.rim_ratio;
    const double floorShare = std::fmin(spec.cutoff_depth_ratio / freshDepth, 1.0);
    const size_t n = work.craters.size();
    count = n;
    RecordCrater* out = place(n);
    if (out == nullptr && n > 0) {
        return TG_ERROR_MEMORY;
    }
    // Blocks of 512 craters on the host threads, each with its own extras, joined in order.
    constexpr size_t kBlock = 512;
    const size_t nblocks = (n + kBlock - 1) / kBlock;
    static thread_local std::vector<std::vector<float>> blockExtras;
    std::vector<std::vector<float>>& blocks = blockExtras;  // the caller's (see generate_into)
    if (blocks.size() < nblocks) {
        blocks.resize(nblocks);
    }
    parallel_for(nblocks, threads, [&](size_t b) {
        std::vector<float>& values = blocks[b];
        values.clear();
        const size_t end = std::min(n, (b + 1) * kBlock);
        for (size_t q = b * kBlock; q < end; ++q) {
            const Crater& c = work.craters[q];
            // FreshnessDegradation::State with constant fresh morphometry and uniform ages.
            const double remaining = std::clamp(1.0 - c.age / spec.lifetime_gyr, 0.0, 1.0);
            const double erosion = floorShare + (1.0 - floorShare) * remaining;
            RecordCrater& r = out[q];
            r = RecordCrater{c.x, c.y, c.diameter, c.age, erosion, c.id,
                             uint32_t(values.size()), 0u, 0u, 0u, 0u};
            const bool terraced = c.diameter >= setup.terraces.onset;  // else none drawn
            const bool complex = setup.profile.is_complex(c.diameter);
            if (!setup.irregular || (!terraced && !complex)) {
                continue;
            }
            // AppendKernelTerraces, then AppendKernelPeaks (crater_kernel.cpp:592-593) into a
            // scratch record: only their counts matter, the offsets are the device's.
            CraterRecord scratch{};
            const size_t start = values.size();
            append_terraces(setup.terraces, terraceSeed, setup.profile, c.diameter, c.id,
                            freshDepth, freshRim, erosion * freshDepth, erosion * freshRim,
                            scratch, values);
            r.terraceCount = uint16_t(scratch.terraceCount);
            r.terraceFloats = uint32_t(values.size() - start);
            if (complex) {
                append_peaks(setup.peaks, peakSeed, c.id, freshDepth, erosion * freshDepth, scratch,
                             values);
                r.peakCount = uint16_t(scratch.peakCount);
            }
            r.extraFloats = uint32_t(values.size() - start);
        }
    });
    std::vector<size_t> base(nblocks + 1, 0);
    for (size_t b = 0; b < nblocks; ++b) {
        base[b + 1] = base[b] + blocks[b].size();
    }
    if (base.back() >= (size_t(1) << 32)) {
        return TG_ERROR_UNSUPPORTED;
    }
    extras.resize(base.back());
    parallel_for(nblocks, threads, [&](size_t b) {
        std::copy(blocks[b].begin(), blocks[b].end(), extras.begin() + base[b]);
        const size_t end = std::min(n, (b + 1) * kBlock);
        for (size_t q = b * kBlock; q < end; ++q) {
            out[q].extraOffset += uint32_t(base[b]);
        }
    });
    return TG_OK;
}

}  // namespace host
}  // namespace tgb

using namespace tgb;
using namespace tgb::host;

namespace {
thread_local std::string g_population_error;

bool same_population(const tg_crater_population& a, const tg_crater_population& b) {
    return a.seed == b.seed && a.sfd_coefficient == b.sfd_coefficient &&
           a.sfd_exponent == b.sfd_exponent && a.min_diameter == b.min_diameter &&
           a.max_diameter == b.max_diameter && a.lifetime_gyr == b.lifetime_gyr &&
           a.depth_ratio == b.depth_ratio && a.rim_ratio == b.rim_ratio &&
           a.cutoff_depth_ratio == b.cutoff_depth_ratio &&
           a.cell_size_factor == b.cell_size_factor && a.margin_radii == b.margin_radii &&
           a.min_resolved_diameter == b.min_resolved_diameter;
}

bool same_shaping(const tg_crater_shaping& a, const tg_crater_shaping& b) {
    return a.profile == b.profile && a.irregular == b.irregular &&
           a.transition_diameter == b.transition_diameter && a.terrace_onset == b.terrace_onset &&
           a.terrace_full == b.terrace_full && a.terrace_min_freshness == b.terrace_min_freshness;
}

bool same_grid(const tg_grid& a, const tg_grid& b) {
    return a.width == b.width && a.height == b.height && a.origin_x == b.origin_x &&
           a.pixel_width == b.pixel_width && a.row_rotation == b.row_rotation &&
           a.origin_y == b.origin_y && a.col_rotation == b.col_rotation &&
           a.pixel_height == b.pixel_height;
}

// The batch a size query built, for the fill call that follows it.
struct BatchCache {
    bool valid = false;
    tg_crater_population spec{};
    tg_crater_shaping shaping{};
    tg_grid grid{};
    std::vector<RecordBlock> blocks;

    bool take(const tg_crater_population& p, const tg_crater_shaping& s, const tg_grid& g,
              std::vector<RecordBlock>& out) {
        const bool hit =
            valid && same_population(spec, p) && same_shaping(shaping, s) && same_grid(grid, g);
        if (hit) {
            out.swap(blocks);
        }
        valid = false;
        blocks = {};
        return hit;
    }

    void keep(const tg_crater_population& p, const tg_crater_shaping& s, const tg_grid& g,
              std::vector<RecordBlock>& in) {
        valid = true;
        spec = p;
        shaping = s;
        grid = g;
        blocks.swap(in);
    }
};
}

extern "C" {

void tg_set_host_threads(unsigned threads) {
    g_host_threads.store(threads);
}

int tg_crater_generate(const tg_crater_population* spec, const double* region, double* x,
                         double* y, double* diameter, double* age, uint64_t* id, size_t capacity,
                         size_t* count) {
    if (spec == nullptr || region == nullptr || count == nullptr) {
        return TG_ERROR_ARGUMENT;
    }
    if (!(spec->min_diameter > 0.0) || !(spec->max_diameter > spec->min_diameter) ||
        !std::isfinite(spec->max_diameter) || !(spec->sfd_coefficient > 0.0) ||
        !(spec->sfd_exponent > 0.0) || !(spec->lifetime_gyr > 0.0) ||
        !(spec->cell_size_factor > 0.0) || !(region[2] >= region[0]) ||
        !(region[3] >= region[1])) {
        return TG_ERROR_ARGUMENT;
    }
    const std::vector<Crater> craters =
        generate(*spec, Box{region[0], region[1], region[2], region[3]},
                 PowerLaw{spec->sfd_coefficient, spec->sfd_exponent});
    *count = craters.size();
    for (size_t n = 0; n < craters.size() && n < capacity; ++n) {
        if (x) x[n] = craters[n].x;
        if (y) y[n] = craters[n].y;
        if (diameter) diameter[n] = craters[n].diameter;
        if (age) age[n] = craters[n].age;
        if (id) id[n] = craters[n].id;
    }
    return TG_OK;
}

int tg_boulder_generate(const tg_boulder_population* spec, const double* region, double spacing,
                        tg_boulder* out, size_t capacity, size_t* count) {
    if (spec == nullptr || region == nullptr || count == nullptr) {
        return TG_ERROR_ARGUMENT;
    }
    const tg_boulder_population& b = *spec;
    if (!(b.min_diameter > 0.0) || !(b.max_diameter > b.min_diameter) ||
        !std::isfinite(b.max_diameter) || !(b.sfd_coefficient > 0.0) ||
        !(b.sfd_exponent > 0.0) || !(b.cell_size_factor > 0.0) || !(spacing > 0.0) ||
        !(b.fade_start_samples >= 0.0) || !(b.fade_end_samples > b.fade_start_samples) ||
        !(region[2] >= region[0]) || !(region[3] >= region[1])) {
        return TG_ERROR_ARGUMENT;
    }
    // ScatterBoulderCandidates (boulder_layer.cpp:263-295): craters of the candidate sizes
    // (BoulderCandidates: the sizes weighted by the richest background abundance, 1 without
    // patches, clusters, maps or bedrock) in the candidate substream, reaching the region by a
    // dome's own margin of 1 radius, bands below the fade's start skipped (BoulderRecords,
    // boulder_layer.cpp:370-374).
    tg_crater_population p{};
    p.seed = substream_seed(b.seed, kBoulderCandidateStream);
    p.min_diameter = b.min_diameter;
    p.max_diameter = b.max_diameter;
    p.lifetime_gyr = 1.0;
    p.cell_size_factor = b.cell_size_factor;
    p.margin_radii = 1.0;
    p.min_resolved_diameter = b.fade_start_samples * spacing;
    const PowerLaw sizes{b.sfd_coefficient, b.sfd_exponent};
    const PowerLaw candidates{b.sfd_coefficient, b.sfd_exponent, 1.0};
    const std::vector<Crater> drawn =
        generate(p, Box{region[0], region[1], region[2], region[3]}, candidates, host_threads());
    // Each part of 4096 candidates thinned on the host threads; the kept joined in order.
    constexpr size_t kPart = 4096;
    const size_t parts = (drawn.size() + kPart - 1) / kPart;
    std::vector<std::vector<tg_boulder>> kept(parts);
    parallel_for(parts, host_threads(), [&](size_t part) {
        const size_t end = std::min(drawn.size(), (part + 1) * kPart);
        for (size_t q = part * kPart; q < end; ++q) {
            const Crater& c = drawn[q];
            const uint32_t low = uint32_t(c.id), high = uint32_t(c.id >> 32);
            // Thin (boulder_layer.cpp:345-358): kept when a draw falls below the background density
            // over the candidates' (1 here: the background abundance is 1 everywhere).
            Stream keep(b.seed, kBoulderAttributeStream, low, high, 0u /* Keep */);
            const double density = 1.0 * sizes.incremental(c.diameter);
            if (keep.next_double() >= density / candidates.incremental(c.diameter)) {
                continue;
            }
            // DrawPose and Wear (boulder_pose.cpp:28-77): height ratio, then wear (its own stream),
            // then the buried share, each uniform between its bounds.
            Stream pose(b.seed, kBoulderAttributeStream, low, high, 1u /* Pose */);
            const double ratio =
                b.min_height_ratio + (b.max_height_ratio - b.min_height_ratio) * pose.next_double();
            Stream wear(b.seed, kBoulderAttributeStream, low, high, 2u /* Wear */);
            wear.next_double();
            wear.next_double();
            const double share = pose.next_double();
            const double burial = b.min_burial + (b.max_burial - b.min_burial) * share;
            const double height = ratio * c.diameter;
            // Drawn into the heights when its resolution weight is positive (boulder_relief.cpp:
            // 298-302, the default relief range holding every boulder that is not a model).
            const double weight = resolution_weight(c.diameter, spacing, b.fade_start_samples,
                                                    b.fade_end_samples);
            if (!(weight > 0.0)) {
                continue;
            }
            kept[part].push_back(tg_boulder{c.x, c.y, c.diameter, height * (1.0 - burial), weight});
        }
    });
    size_t n = 0;
    for (const std::vector<tg_boulder>& list : kept) {
        for (const tg_boulder& stone : list) {
            if (out != nullptr && n < capacity) {
                out[n] = stone;
            }
            ++n;
        }
    }
    *count = n;
    return TG_OK;
}

int tg_crater_batch(const tg_crater_population* spec, const tg_crater_shaping* shaping,
                    const tg_grid* grid, void* kernel, void* records, size_t record_capacity,
                    float* data, size_t data_capacity, double* footprints, size_t* n_records,
                    size_t* n_data) {
    if (spec == nullptr || shaping == nullptr || grid == nullptr || n_records == nullptr ||
        n_data == nullptr) {
        return TG_ERROR_ARGUMENT;
    }
    BatchSetup setup;
    if (int st = batch_setup(*spec, *shaping, *grid, setup)) {
        return st;
    }
    const LayerProfile& profile = setup.profile;
    const TerraceOptions& terraces = setup.terraces;
    const PeakOptions& peaks = setup.peaks;
    const double spacing = setup.spacing;
    const bool irregular = setup.irregular;
    const double reachRadii = setup.reachRadii;
    // A call that asks only for the sizes keeps what it built, and the next call from the same
    // thread with the same inputs copies that out instead of building it again.
    std::vector<RecordBlock> blocks;
    const unsigned threads = host_threads();
    static thread_local BatchCache cache;
    // The calling thread's working arrays, kept from call to call (named by reference: the loop
    // bodies run on other threads).
    static thread_local BatchWork workspace;
    BatchWork& work = workspace;
    if (!cache.take(*spec, *shaping, *grid, blocks)) {
        if (int st = batch_order(setup, *grid, threads, work)) {
            return st;
        }
        const std::vector<Crater>& craters = work.craters;
        const std::vector<uint32_t>& sorted = work.sorted;
        const std::vector<uint32_t>& order = sorted;

        // SeededCraterApply (apply_options.cpp:57): every per-crater stream follows the layer seed.
        const uint32_t irregularitySeed = substream_seed(spec->seed, kCraterIrregularityStream);
        const uint32_t noiseSeed = substream_seed(spec->seed, kCraterNoiseStream);
        const uint32_t terraceSeed = substream_seed(spec->seed, kCraterTerraceStream);
        const uint32_t peakSeed = substream_seed(spec->seed, kCraterPeakStream);
        const uint32_t textureSeed = substream_seed(spec->seed, kCraterTextureStream);
        const uint32_t textureKeySeed = substream_seed(textureSeed, kCraterTextureStream);

        auto build = [&](const Crater& c, RecordBlock& block, const uint32_t* words) {
            std::vector<CraterRecord>& out = block.records;
            std::vector<float>& values = block.values;
            std::vector<double>& foot = block.foot;
            const double resolution = resolution_weight(c.diameter, spacing);
            if (resolution == 0.0) {
                return;
            }
            const Outline outline = irregular ? irregular_outline(words) : Outline{};
            // CratersOnRaster: the footprint window must hold a cell of the grid.
            double scale = 1.0;
            for (int k = 0; k < outline.harmonics; ++k) {
                scale += std::fabs(outline.amplitudes[k]);
            }
            scale *= std::sqrt(outline.ellipticity);
            const double reach = scale * reachRadii * (0.5 * c.diameter);
            if (!footprint_cells(*grid, c.x, c.y, reach)) {
                return;
            }
            // FreshnessDegradation::State with constant fresh morphometry and uniform ages.
            const double freshDepth = spec->depth_ratio, freshRim = spec->rim_ratio;
            const double floorShare = std::fmin(spec->cutoff_depth_ratio / freshDepth, 1.0);
            const double remaining = std::clamp(1.0 - c.age / spec->lifetime_gyr, 0.0, 1.0);
            const double erosion = floorShare + (1.0 - floorShare) * remaining;
            CraterRecord r{};
            r.diameter = float(c.diameter);
            r.freshDepth = float(freshDepth);
            r.freshRim = float(freshRim);
            r.currentDepth = float(erosion * freshDepth);
            r.currentRim = float(erosion * freshRim);
            r.diffusion = 0.0f;
            r.resolution = float(resolution);
            r.noiseKey = crater_key(c.id, noiseSeed);
            r.textureKey = crater_key(c.id, textureKeySeed);
            r.x = float(c.x);
            r.xLow = float(c.x - double(r.x));
            r.y = float(c.y);
            r.yLow = float(c.y - double(r.y));
            r.ellipticity = float(outline.ellipticity);
            r.heading = float(outline.heading);
            r.harmonicOffset = uint32_t(values.size());
            r.firstHarmonic = uint32_t(outline.firstHarmonic);
            r.harmonicCount = uint32_t(outline.harmonics);
            for (int k = 0; k < outline.harmonics; ++k) {
                values.push_back(float(outline.amplitudes[k]));
                values.push_back(float(outline.phases[k]));
            }
            r.tableCount = 0;
            r.tableOffset = uint32_t(values.size());
            r.markCount = 0;
            r.markOffset = uint32_t(values.size());
            if (irregular) {
                // AppendKernelTerraces, then AppendKernelPeaks (MakeCraterKernelBatch,
                // crater_kernel.cpp:592-593); peaks only on complex craters.
                append_terraces(terraces, terraceSeed, profile, c.diameter, c.id, freshDepth,
                                freshRim, erosion * freshDepth, erosion * freshRim, r, values);
                if (profile.is_complex(c.diameter)) {
                    append_peaks(peaks, peakSeed, c.id, freshDepth, erosion * freshDepth, r, values);
                }
            }
            out.push_back(r);
            foot.push_back(c.x);
            foot.push_back(c.y);
            foot.push_back(reach);
        };
        constexpr size_t kBlock = 512;
        const size_t nblocks = (order.size() + kBlock - 1) / kBlock;
        blocks.swap(work.blocks);  // the blocks' vectors keep their memory from the last batch
        blocks.resize(nblocks);
        parallel_for(nblocks, threads, [&](size_t b) {
            const size_t begin = b * kBlock, end = std::min(order.size(), (b + 1) * kBlock);
            blocks[b].records.clear();
            blocks[b].values.clear();
            blocks[b].foot.clear();
            // The block's outline draws first, all its craters' streams at once (the words in
            // the running thread's own scratch).
            static thread_local std::vector<uint32_t> words;
            if (irregular) {
                uint64_t ids[kBlock];
                for (size_t q = begin; q < end; ++q) {
                    ids[q - begin] = craters[order[q]].id;
                }
                outline_words(ids, end - begin, irregularitySeed, words);
            }
            for (size_t q = begin; q < end; ++q) {
                build(craters[order[q]], blocks[b],
                      irregular ? words.data() + (q - begin) * 4 * kOutlineBlocks : nullptr);
            }
        });
    }
    // Where each block lands in the outputs: records and footprints in order, data offsets moved
    // by the data before (an empty batch still hands the kernel one data float, 0).
    std::vector<size_t> recordBase(blocks.size() + 1, 0), dataBase(blocks.size() + 1, 0);
    for (size_t b = 0; b < blocks.size(); ++b) {
        recordBase[b + 1] = recordBase[b] + blocks[b].records.size();
        dataBase[b + 1] = dataBase[b] + blocks[b].values.size();
    }
    const size_t nRecords = recordBase.back();
    const size_t nValues = std::max<size_t>(dataBase.back(), 1);
    const bool query = records == nullptr && data == nullptr && footprints == nullptr;
    *n_records = nRecords;
    *n_data = nValues;
    if (kernel != nullptr) {
        batch_shape_kernel(setup, kernel);
    }
    if (records != nullptr && record_capacity < nRecords) {
        return TG_ERROR_ARGUMENT;
    }
    if (data != nullptr && data_capacity < nValues) {
        return TG_ERROR_ARGUMENT;
    }
    const bool withFoot = footprints != nullptr && record_capacity >= nRecords;
    if (!query) {
        // Each block's records, data and footprints copied to their place on the host threads.
        parallel_for(blocks.size(), threads, [&](size_t b) {
            const RecordBlock& block = blocks[b];
            const uint32_t base = uint32_t(dataBase[b]);
            if (records != nullptr) {
                CraterRecord* dst = static_cast<CraterRecord*>(records) + recordBase[b];
                for (size_t i = 0; i < block.records.size(); ++i) {
                    CraterRecord r = block.records[i];
                    r.harmonicOffset += base;
                    r.tableOffset += base;
                    r.markOffset += base;
                    if (r.terraceCount > 0u) {
                        r.terraceOffset += base;
                    }
                    if (r.peakCount > 0u) {
                        r.peakOffset += base;
                    }
                    dst[i] = r;
                }
            }
            if (data != nullptr && !block.values.empty()) {
                std::memcpy(data + base, block.values.data(), block.values.size() * sizeof(float));
            }
            if (withFoot && !block.foot.empty()) {
                std::memcpy(footprints + 3 * recordBase[b], block.foot.data(),
                            block.foot.size() * sizeof(double));
            }
        });
        if (data != nullptr && dataBase.back() == 0) {
            data[0] = 0.0f;
        }
    }
    if (query) {
        cache.keep(*spec, *shaping, *grid, blocks);
    } else {
        work.blocks.swap(blocks);
    }
    return TG_OK;
}

}  // extern "C"
