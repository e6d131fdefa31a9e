// Oracle harness: the reference TerrainGen pipeline behind a small C ABI, for tests only.
//
// Built three ways by oracle/Makefile, all from the reference's own sources:
//   libtgref.so         - the reference CPU path (`tgref_evaluate` with backend 0);
//   libtgref_capture.so - the reference pipeline with Backend::Cuda routed through the product's
//                         drop-in CudaCompute (terraingen_b200/adapter/cuda_compute.cpp), whose
//                         tg_* calls land in the capture stubs below: they record exactly what
//                         the reference hands its GPU backend (kernel bytes, crater records,
//                         tile lists, positions) and leave the heights as they were. Runs
//                         without a GPU; tests/golden/make_fixtures.py stores the captures;
//   libtgref_cuda.so    - the same pipeline with the adapter linked to libtgb200.so, so
//                         Backend::Cuda runs the product's kernels inside the reference's
//                         Terrain::Evaluate (GPU parity tests).
#include "terraingen/terraingen.h"

#include "terraingen/distribution/power_law.h"
#include "terraingen/layers/craters/degradation/diffusion.h"
#include "terraingen/layers/craters/degradation/diffusivities.h"
#include "terraingen/layers/craters/degradation/freshness_degradation.h"
#include "terraingen/layers/craters/profiles/complex.h"
#include "terraingen/layers/craters/profiles/fassett_thomson.h"
#include "terraingen/layers/craters/profiles/martin_parkes_dunstan.h"
#include "terraingen/layers/craters/shaping/morphometry.h"
#include "terraingen/layers/boulders/boulder_layer.h"
#include "terraingen/layers/fade.h"
#include "terraingen/layers/kernels/craters.h"
#include "terraingen/sources/diamond_square.h"
#include "terraingen/sources/raster_source.h"
#include "terraingen/sources/source_chain.h"

#include "sources/seam_field.h"
#include "terraingen/util/log.h"

#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#ifdef TGREF_HOOKS
#include "tgb200_hooks.h"
#endif

using namespace terraingen;

namespace {

thread_local std::string g_error;

}  // namespace

extern "C" {

/// One scene: a grid, a source and up to one noise layer and one crater layer.
struct tgref_scene {
    uint32_t width, height;
    double transform[6];  // GDAL order: origin x, pixel width, 0, origin y, 0, pixel height
    // source: 0 flat, 1 synthetic fractal stack
    int32_t source;
    float elevation;
    uint32_t sourceFractals;
    Fractal sourceStack[8];
    // noise layer (none when 0 fractals)
    uint32_t layerFractals;
    Fractal layerStack[8];
    // crater layer (none when craters == 0)
    int32_t craters;
    uint32_t seed;
    double sfdCoefficient, sfdExponent, minDiameter, maxDiameter;
    double lifetimeGyr, depthRatio, rimRatio;
    // 0 Fassett-Thomson, 1 Martin-Parkes-Dunstan, 2 complex over FT (lunar shape with
    // transitionDiameter), 3 diffused MPD with matched diffusion (the reference's default models)
    int32_t profile;
    double transitionDiameter;
    // 0 DefaultCraterApply (irregular outlines, terraces, peaks), 1 plain CraterApplyOptions
    int32_t applyPreset;
    double noiseAmplitude, rimNoiseAmplitude, wallStreaks, ejecta, rimSigma;
    double terraceOnset, terraceFull;
    // boulder layer (none when boulders == 0): sizes N(>D) = c D^-exponent per m^2 on
    // [min, max], height ratio fixed, no burial
    int32_t boulders;
    uint32_t boulderSeed;
    double boulderCoefficient, boulderExponent, boulderMin, boulderMax, heightRatio;
    // crater datums: 0 none, 1 plane, 2 mean height, 3 center height (CraterDatum), and the
    // share of the interior they replace
    int32_t datum;
    double interiorReplacement;
    // a sphere of this radius (m) when positive, the grid's transform then in degrees of
    // longitude and latitude; a plane when 0
    double bodyRadius;
    // CraterTerraces::minFreshness when positive (with terraceOnset); the default 0.3 otherwise
    double terraceMinFreshness;
};

const char* tgref_error() {
    return g_error.c_str();
}

/// How many times the drop-in build's hooks at the CPU-only stages ran on the device (0 in the
/// other builds).
long tgref_hook_calls() {
#ifdef TGREF_HOOKS
    return tgb200_hook_calls();
#else
    return 0;
#endif
}

}  // extern "C"

namespace {

std::vector<Fractal> Stack(const Fractal* fractals, uint32_t count) {
    return std::vector<Fractal>(fractals, fractals + count);
}

std::shared_ptr<CraterLayer> MakeCraterLayer(const tgref_scene& s, TerrainBase base = {}) {
    auto density = std::make_shared<PowerLawSfd>(s.sfdCoefficient, s.sfdExponent, SfdKind::Density,
                                                  DiameterRange{s.minDiameter, s.maxDiameter});
    CraterModels models;
    models.density = density;
    const double depth = s.depthRatio, rim = s.rimRatio;
    FreshMorphometry fresh = [depth, rim](double) { return CraterMorphometry{depth, rim}; };
    if (s.profile == 3) {
        // The reference's default models (steady-state ages, matched diffusion of diffused MPD
        // profiles) on the scene's density.
        CraterModels defaults = DefaultCraterModels();
        defaults.density = density;
        models = defaults;
    } else {
        auto ages = std::make_shared<UniformAges>(s.lifetimeGyr);
        models.ages = ages;
        models.degradation = std::make_shared<FreshnessDegradation>(ages, fresh);
        std::shared_ptr<const CraterProfile> simple;
        if (s.profile == 1) {
            simple = std::make_shared<MartinParkesDunstanProfile>();
        } else {
            simple = std::make_shared<FassettThomsonProfile>();
        }
        if (s.profile == 2) {
            ComplexCraterShape shape = LunarComplexCraterShape();
            shape.transitionDiameter = s.transitionDiameter;
            models.profile = std::make_shared<ComplexCraterProfile>(simple, shape);
        } else {
            models.profile = simple;
        }
    }
    CraterLayerOptions options;
    options.seed = s.seed;
    options.generation.minDiameter = s.minDiameter;
    options.generation.maxDiameter = s.maxDiameter;
    if (s.applyPreset == 1) {
        options.apply = CraterApplyOptions{};
    }
    options.apply.noise.amplitude = s.noiseAmplitude;
    options.apply.noise.rimAmplitude = s.rimNoiseAmplitude;
    options.apply.texture.wallStreaks = s.wallStreaks;
    options.apply.texture.ejecta = s.ejecta;
    options.apply.rimSmoothing.sigmaRadii = s.rimSigma;
    if (s.datum > 0) {
        options.apply.datum = static_cast<CraterDatum>(s.datum);
        options.apply.interiorReplacement = s.interiorReplacement;
    }
    if (s.terraceOnset > 0.0) {
        options.apply.terraces.onsetDiameter = s.terraceOnset;
        options.apply.terraces.fullDiameter = s.terraceFull;
        if (s.terraceMinFreshness > 0.0) {
            options.apply.terraces.minFreshness = s.terraceMinFreshness;
        }
    }
    return std::make_shared<CraterLayer>(std::move(models), std::move(options), std::move(base));
}

std::shared_ptr<BoulderLayer> MakeBoulderLayer(const tgref_scene& s) {
    BoulderLayerOptions options;
    options.seed = s.boulderSeed;
    options.sizes.distribution = std::make_shared<PowerLawSfd>(
        s.boulderCoefficient, s.boulderExponent, SfdKind::Density,
        DiameterRange{s.boulderMin, s.boulderMax});
    options.sizes.minDiameter = s.boulderMin;
    options.sizes.maxDiameter = s.boulderMax;
    options.pose.minHeightRatio = s.heightRatio;
    options.pose.maxHeightRatio = s.heightRatio;
    options.pose.minBurial = 0.0;
    options.pose.maxBurial = 0.0;
    return std::make_shared<BoulderLayer>(options);
}

Terrain MakeTerrain(const tgref_scene& s, bool withBoulders = true) {
    std::shared_ptr<const Source> source;
    if (s.bodyRadius > 0.0) {
        // A flat site on a sphere: the grid in degrees, the craters on the body.
        const Surface surface = Surface::Sphere(s.bodyRadius);
        const Vec2d center{s.transform[0] + 0.5 * s.width * s.transform[1],
                           s.transform[3] + 0.5 * s.height * s.transform[5]};
        source = std::make_shared<FlatSource>(s.width, s.height,
                                              std::fabs(s.transform[1]) * surface.UnitLength(),
                                              s.elevation, center, surface);
        std::vector<LayerPtr> layers;
        if (s.craters != 0) {
            layers.push_back(MakeCraterLayer(s, TerrainBase{surface, source}));
        }
        return Terrain(surface, source, layers);
    }
    if (s.source == 1) {
        source = std::make_shared<SyntheticSource>(Stack(s.sourceStack, s.sourceFractals),
                                                   s.elevation);
    } else {
        source = std::make_shared<FlatSource>(s.width, s.height,
                                              std::fabs(s.transform[1]), s.elevation);
    }
    std::vector<LayerPtr> layers;
    if (s.layerFractals > 0) {
        NoiseLayerOptions options;
        options.fractals = Stack(s.layerStack, s.layerFractals);
        options.sourceResolvesPixels = std::nullopt;
        layers.push_back(std::make_shared<NoiseLayer>(options));
    }
    if (s.craters != 0) {
        layers.push_back(MakeCraterLayer(s));
    }
    if (s.boulders != 0 && withBoulders) {
        layers.push_back(MakeBoulderLayer(s));
    }
    return Terrain(Surface{}, source, layers);
}

}  // namespace

extern "C" {

/// Evaluates the scene's grid on the CPU (backend 0) or on Backend::Cuda (backend 1) with
/// `threads` threads (0: every core); heights into `out` (width x height floats). `ms` gets the
/// wall time of the evaluation alone. Returns 0, or -1 with tgref_error() set.
int tgref_evaluate(const tgref_scene* s, int backend, unsigned threads, float* out, double* ms) {
    try {
        SetLogLevel(LogLevel::Warning);
        const Terrain terrain = MakeTerrain(*s);
        const GeoTransform transform = GeoTransform::FromGdal(
            {s->transform[0], s->transform[1], s->transform[2], s->transform[3], s->transform[4],
             s->transform[5]});
        const RasterGrid grid{s->width, s->height, transform};
        EvaluationOptions options;
        options.threads = threads;
        options.backend = backend == 1 ? Backend::Cuda : Backend::Cpu;
#ifdef TGREF_HOOKS
        // The drop-in build's hooks at the CPU-only stages follow the evaluation's backend.
        tgb200_set_hooks_active(backend == 1);
#endif
        const auto t0 = std::chrono::steady_clock::now();
        const Raster<float> heights = terrain.Evaluate(grid, options);
        const auto t1 = std::chrono::steady_clock::now();
        if (ms != nullptr) {
            *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        std::memcpy(out, heights.Values().data(), heights.Values().size() * sizeof(float));
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// The scene's heights at `n` points (x, y pairs) through the reference's point path:
/// Terrain::HeightsAt (Source::HeightsAt, src/pipeline/terrain.cpp:133-154: EvaluatePoints, the
/// points in Morton-ordered batches of nearby points, each batch's layers prepared over its own
/// area) at sample `spacing`. Returns 0, or -1 with tgref_error() set.
int tgref_points(const tgref_scene* s, const double* xy, uint32_t n, double spacing, float* out) {
    try {
        SetLogLevel(LogLevel::Warning);
        const Terrain terrain = MakeTerrain(*s);
        std::vector<Vec2d> points(n);
        for (uint32_t i = 0; i < n; ++i) {
            points[i] = Vec2d{xy[2 * size_t(i)], xy[2 * size_t(i) + 1]};
        }
        terrain.HeightsAt(Span<const Vec2d>(points), Span<float>(out, n), spacing);
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// The number of craters the scene's crater layer generates over `region`
/// (x0, y0, x1, y1 in meters), and their centers, diameters and ids into the arrays when given
/// (capacity `n`).
long tgref_craters(const tgref_scene* s, const double* region, double spacing, double* x,
                   double* y, double* diameter, double* age, uint64_t* id, long n) {
    try {
        SetLogLevel(LogLevel::Warning);
        const auto layer = MakeCraterLayer(*s);
        const CraterList list =
            layer->Craters({region[0], region[1], region[2], region[3]}, spacing);
        const long count = static_cast<long>(list.Size());
        for (long i = 0; i < count && i < n; ++i) {
            const Crater c = list.At(static_cast<std::size_t>(i));
            if (x) x[i] = c.x;
            if (y) y[i] = c.y;
            if (diameter) diameter[i] = c.diameter;
            if (age) age[i] = c.ageGyr;
            if (id) id[i] = c.id;
        }
        return count;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// The boulders the scene's boulder layer draws into its grid as domes, as its ApplySamples picks
/// them (boulder_relief.cpp:298-302, 372-425): placed over the grid's bounds grown by half a
/// sample, on the ground of the layers below, drawn when their relief range holds them and their
/// resolution weight is positive. Per boulder: x, y, diameter, exposed height, weight (5 doubles)
/// into `out` (capacity `n` boulders); returns the count, or -1.
long tgref_boulders(const tgref_scene* s, double* out, long n) {
    try {
        SetLogLevel(LogLevel::Warning);
        const auto layer = MakeBoulderLayer(*s);
        const Terrain below = MakeTerrain(*s, false);
        const GeoTransform transform = GeoTransform::FromGdal(
            {s->transform[0], s->transform[1], s->transform[2], s->transform[3], s->transform[4],
             s->transform[5]});
        const RasterGrid grid{s->width, s->height, transform};
        const double spacing = std::fabs(s->transform[1]);
        const Bounds2d bounds = grid.Bounds().Expanded(0.5 * spacing);
        const BoulderList list = layer->Boulders(bounds, spacing, &below);
        const BoulderLayerOptions& options = layer->Options();
        long count = 0;
        for (std::size_t i = 0; i < list.Size(); ++i) {
            const Boulder b = list.At(i);
            const double weight = ResolutionWeight(b.diameter, spacing, options.fade);
            if (!options.rendering.reliefRange.Holds(b.diameter, b.model) || weight <= 0.0) {
                continue;
            }
            if (count < n && out != nullptr) {
                double* o = out + 5 * count;
                o[0] = b.x;
                o[1] = b.y;
                o[2] = b.diameter;
                o[3] = b.ExposedHeight();
                o[4] = weight;
            }
            ++count;
        }
        return count;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// tgref_boulders with the pose drawn between bounds: height ratio in [pose[0], pose[1]] and
/// buried share in [pose[2], pose[3]] (BoulderPose).
long tgref_boulders_posed(const tgref_scene* s, const double* pose, double* out, long n) {
    try {
        SetLogLevel(LogLevel::Warning);
        BoulderLayerOptions options = MakeBoulderLayer(*s)->Options();
        options.pose.minHeightRatio = pose[0];
        options.pose.maxHeightRatio = pose[1];
        options.pose.minBurial = pose[2];
        options.pose.maxBurial = pose[3];
        const auto layer = std::make_shared<BoulderLayer>(options);
        const GeoTransform transform = GeoTransform::FromGdal(
            {s->transform[0], s->transform[1], s->transform[2], s->transform[3], s->transform[4],
             s->transform[5]});
        const RasterGrid grid{s->width, s->height, transform};
        const double spacing = std::fabs(s->transform[1]);
        const BoulderList list = layer->Boulders(grid.Bounds().Expanded(0.5 * spacing), spacing,
                                                 nullptr);
        long count = 0;
        for (std::size_t i = 0; i < list.Size(); ++i) {
            const Boulder b = list.At(i);
            const double weight = ResolutionWeight(b.diameter, spacing, options.fade);
            if (!options.rendering.reliefRange.Holds(b.diameter, b.model) || weight <= 0.0) {
                continue;
            }
            if (count < n && out != nullptr) {
                double* o = out + 5 * count;
                o[0] = b.x;
                o[1] = b.y;
                o[2] = b.diameter;
                o[3] = b.ExposedHeight();
                o[4] = weight;
            }
            ++count;
        }
        return count;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// The reference's DiamondSquareUpsampler over `posts` (pw x ph floats on `postTransform`), read at
/// the cells of an `ow` x `oh` grid on `outTransform`, through a RasterSource in a Terrain: the
/// heights into `out`, the evaluation's wall time into `ms`.
int tgref_ds_on(int backend, const float* posts, uint32_t pw, uint32_t ph,
                const double* postTransform, double fractalDimension, double scale, int interp,
                uint32_t seed, uint32_t ow, uint32_t oh, const double* outTransform,
                unsigned threads, float* out, double* ms);

int tgref_ds(const float* posts, uint32_t pw, uint32_t ph, const double* postTransform,
             double fractalDimension, double scale, int interp, uint32_t seed, uint32_t ow,
             uint32_t oh, const double* outTransform, unsigned threads, float* out, double* ms) {
    return tgref_ds_on(0, posts, pw, ph, postTransform, fractalDimension, scale, interp, seed,
                       ow, oh, outTransform, threads, out, ms);
}

/// tgref_ds on Backend::Cpu (backend 0) or Backend::Cuda (1; in the drop-in build the
/// refinement then runs through libtgb200's hook).
int tgref_ds_on(int backend, const float* posts, uint32_t pw, uint32_t ph,
                const double* postTransform, double fractalDimension, double scale, int interp,
                uint32_t seed, uint32_t ow, uint32_t oh, const double* outTransform,
                unsigned threads, float* out, double* ms) {
    try {
        SetLogLevel(LogLevel::Warning);
        const RasterGrid postGrid{pw, ph,
                                  GeoTransform::FromGdal({postTransform[0], postTransform[1],
                                                          postTransform[2], postTransform[3],
                                                          postTransform[4], postTransform[5]})};
        Raster<float> raster(postGrid);
        std::memcpy(raster.Values().data(), posts, size_t(pw) * ph * sizeof(float));
        DiamondSquareOptions options;
        options.fractalDimension = fractalDimension;
        options.scale = scale;
        options.interp = interp == 1 ? DiamondSquareInterp::CatmullRom : DiamondSquareInterp::Bilinear;
        options.seed = seed;
        RasterSourceOptions sourceOptions;
        sourceOptions.upsampler = std::make_shared<DiamondSquareUpsampler>(options);
        auto source = std::make_shared<RasterSource>(std::move(raster), sourceOptions);
        const Terrain terrain(Surface{}, source, {});
        EvaluationOptions evaluation;
        evaluation.threads = threads;
        evaluation.backend = backend == 1 ? Backend::Cuda : Backend::Cpu;
#ifdef TGREF_HOOKS
        tgb200_set_hooks_active(backend == 1);
#endif
        const RasterGrid grid{ow, oh,
                              GeoTransform::FromGdal({outTransform[0], outTransform[1],
                                                      outTransform[2], outTransform[3],
                                                      outTransform[4], outTransform[5]})};
        const auto t0 = std::chrono::steady_clock::now();
        const Raster<float> heights = terrain.Evaluate(grid, evaluation);
        const auto t1 = std::chrono::steady_clock::now();
        if (ms != nullptr) {
            *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        std::memcpy(out, heights.Values().data(), heights.Values().size() * sizeof(float));
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// Two raster sources on `grid` (GDAL `transform`): `earlier` (NaN where it has no data) and
/// `later`, cubic-upsampled RasterSources as a SourceChain joins them.
struct SeamPair {
    std::shared_ptr<const Source> earlier, later;
    RasterGrid grid;
};

SeamPair MakeSeamPair(const float* earlier, const float* later, uint32_t w, uint32_t h,
                      const double* transform) {
    const RasterGrid grid{w, h, GeoTransform::FromGdal({transform[0], transform[1], transform[2],
                                                        transform[3], transform[4], transform[5]})};
    Raster<float> a(grid), b(grid);
    std::memcpy(a.Values().data(), earlier, size_t(w) * h * sizeof(float));
    std::memcpy(b.Values().data(), later, size_t(w) * h * sizeof(float));
    a.SetNoData(std::numeric_limits<float>::quiet_NaN());
    b.SetNoData(std::numeric_limits<float>::quiet_NaN());
    return SeamPair{std::make_shared<RasterSource>(std::move(a)),
                    std::make_shared<RasterSource>(std::move(b)), grid};
}

ChainSeams MakeSeams(int mode, double width, double decay) {
    ChainSeams seams;
    seams.mode = mode == 1   ? ChainSeamMode::Feather
                 : mode == 2 ? ChainSeamMode::Height
                 : mode == 3 ? ChainSeamMode::Slope
                             : ChainSeamMode::None;
    seams.width = width;
    seams.decayLength = decay;
    return seams;
}

/// The reference's seam between the two sources (detail::BuildSeamField, seam_field.cpp:663):
/// the lattice (SeamLattice) size and GDAL transform, and at each of its posts (at most
/// `capacity`) the samples the solve starts from - 1 where `earlier` has data, `earlier` minus
/// `later` where both do (NaN elsewhere), filled 64 rows at a time as SampleSources does - and
/// the field's value.
int tgref_seam(const float* earlier, const float* later, uint32_t w, uint32_t h,
               const double* transform, int mode, double width, double decay, uint32_t* lw,
               uint32_t* lh, double* latticeTransform, uint8_t* data, float* difference,
               float* field, size_t capacity, double* ms) {
    try {
        SetLogLevel(LogLevel::Warning);
        const SeamPair pair = MakeSeamPair(earlier, later, w, h, transform);
        const ChainSeams seams = MakeSeams(mode, width, decay);
        const RasterGrid lattice = SeamLattice(pair.grid, seams);
        *lw = uint32_t(lattice.width);
        *lh = uint32_t(lattice.height);
        const std::array<double, 6> gdal = lattice.transform.ToGdal();
        for (int i = 0; i < 6; ++i) {
            latticeTransform[i] = gdal[size_t(i)];
        }
        const size_t posts = lattice.width * lattice.height;
        if (posts > capacity) {
            return 1;
        }
        const double spacing = pair.grid.PixelSize();
        for (size_t top = 0; top < lattice.height; top += 64) {
            const size_t rows = std::min<size_t>(64, lattice.height - top);
            GeoTransform t = lattice.transform;
            const Vec2d origin = lattice.transform.PixelToWorld(0.0, double(top));
            t.originX = origin.x;
            t.originY = origin.y;
            Raster<float> above(RasterGrid{lattice.width, rows, t});
            Raster<float> below(RasterGrid{lattice.width, rows, t});
            pair.earlier->Fill(above, spacing);
            pair.later->Fill(below, spacing);
            for (size_t row = 0; row < rows; ++row) {
                for (size_t col = 0; col < lattice.width; ++col) {
                    const float a = above(col, row), b = below(col, row);
                    const size_t k = (top + row) * lattice.width + col;
                    data[k] = above.IsMissing(a) ? 0 : 1;
                    difference[k] =
                        !above.IsMissing(a) && !below.IsMissing(b) && std::isfinite(a) &&
                                std::isfinite(b)
                            ? float(double(a) - double(b))
                            : std::numeric_limits<float>::quiet_NaN();
                }
            }
        }
        const auto t0 = std::chrono::steady_clock::now();
        const detail::SeamField seam =
            detail::BuildSeamField(*pair.earlier, *pair.later, pair.grid, seams);
        const auto t1 = std::chrono::steady_clock::now();
        if (ms != nullptr) {
            *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        for (size_t row = 0; row < lattice.height; ++row) {
            for (size_t col = 0; col < lattice.width; ++col) {
                field[row * lattice.width + col] =
                    seam.Post(std::ptrdiff_t(col), std::ptrdiff_t(row));
            }
        }
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// A SourceChain of the two sources joined by `mode` evaluated on an `ow` x `oh` grid
/// (`outTransform`): the later source plus the seam where the earlier has no data
/// (SourceChain::FillGridGaps, source_chain.cpp:167).
int tgref_chain(const float* earlier, const float* later, uint32_t w, uint32_t h,
                const double* transform, int mode, double width, double decay, uint32_t ow,
                uint32_t oh, const double* outTransform, float* out) {
    try {
        SetLogLevel(LogLevel::Warning);
        const SeamPair pair = MakeSeamPair(earlier, later, w, h, transform);
        auto chain = std::make_shared<SourceChain>(
            std::vector<std::shared_ptr<const Source>>{pair.earlier, pair.later},
            MakeSeams(mode, width, decay));
        const Terrain terrain(Surface{}, chain, {});
        EvaluationOptions evaluation;
        evaluation.threads = 1;
        evaluation.backend = Backend::Cpu;
        const RasterGrid grid{ow, oh,
                              GeoTransform::FromGdal({outTransform[0], outTransform[1],
                                                      outTransform[2], outTransform[3],
                                                      outTransform[4], outTransform[5]})};
        const Raster<float> heights = terrain.Evaluate(grid, evaluation);
        std::memcpy(out, heights.Values().data(), heights.Values().size() * sizeof(float));
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// A SourceChain of `n` raster sources, source k (`widths[k]` x `heights[k]` floats at `rasters[k]`,
/// NaN where it has no data) on its own grid (GDAL transform `transforms[6k..6k+5]`), joined by
/// `mode`, evaluated on an `ow` x `oh` grid: the chain's nested seams as the reference builds
/// them (SourceChain::Seam over BoundedGrid of the source before the last, source_chain.cpp:144).
int tgref_patch_chain(uint32_t n, const float* const* rasters, const uint32_t* widths,
                      const uint32_t* heights, const double* transforms, int mode, double width,
                      double decay, uint32_t ow, uint32_t oh, const double* outTransform,
                      float* out) {
    try {
        SetLogLevel(LogLevel::Warning);
        std::vector<std::shared_ptr<const Source>> sources;
        for (uint32_t k = 0; k < n; ++k) {
            const double* t = transforms + 6 * k;
            const RasterGrid grid{widths[k], heights[k],
                                  GeoTransform::FromGdal({t[0], t[1], t[2], t[3], t[4], t[5]})};
            Raster<float> r(grid);
            std::memcpy(r.Values().data(), rasters[k], size_t(widths[k]) * heights[k] * 4);
            r.SetNoData(std::numeric_limits<float>::quiet_NaN());
            sources.push_back(std::make_shared<RasterSource>(std::move(r)));
        }
        auto chain = std::make_shared<SourceChain>(std::move(sources),
                                                   MakeSeams(mode, width, decay));
        const Terrain terrain(Surface{}, chain, {});
        EvaluationOptions evaluation;
        evaluation.threads = 0;
        evaluation.backend = Backend::Cpu;
        const RasterGrid grid{ow, oh,
                              GeoTransform::FromGdal({outTransform[0], outTransform[1],
                                                      outTransform[2], outTransform[3],
                                                      outTransform[4], outTransform[5]})};
        const Raster<float> result = terrain.Evaluate(grid, evaluation);
        std::memcpy(out, result.Values().data(), result.Values().size() * sizeof(float));
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// The scene's heights without its boulder layer (the base the boulders are drawn on).
int tgref_evaluate_below_boulders(const tgref_scene* s, unsigned threads, float* out) {
    try {
        SetLogLevel(LogLevel::Warning);
        const Terrain terrain = MakeTerrain(*s, false);
        const GeoTransform transform = GeoTransform::FromGdal(
            {s->transform[0], s->transform[1], s->transform[2], s->transform[3], s->transform[4],
             s->transform[5]});
        EvaluationOptions options;
        options.threads = threads;
        options.backend = Backend::Cpu;
        const Raster<float> heights =
            terrain.Evaluate(RasterGrid{s->width, s->height, transform}, options);
        std::memcpy(out, heights.Values().data(), heights.Values().size() * sizeof(float));
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

}  // extern "C"

extern "C" {

/// KernelDatumRelief (the reference's header function, on the CPU) at every point of a lattice
/// strip as crater_datums.slang adds it: `heights` (rows x width) += the relief of target
/// first_row + row at point column, over the index a captured tg_crater_datums call holds.
int tgref_datum_relief(const void* kernel, const void* records, const float* data,
                       const float* bandFloats, const uint32_t* bandCells, const uint32_t* cells,
                       const uint32_t* entries, const uint32_t* targets, uint32_t width,
                       uint32_t rows, uint32_t firstRow, float* heights) {
    try {
        CraterDatumKernel k;
        std::memcpy(&k, kernel, sizeof(k));
        const auto* recs = static_cast<const CraterRecord*>(records);
        CraterData values;
        values.values = data;
        for (uint32_t r = 0; r < rows; ++r) {
            for (uint32_t p = 0; p < width; ++p) {
                float& h = heights[size_t(r) * width + p];
                h = h + KernelDatumRelief(k, values, recs, bandFloats, bandCells, cells, entries,
                                          targets[firstRow + r], p);
            }
        }
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

}  // extern "C"

#include "terraingen/raster/geotiff/geotiff.h"
#include "terraingen/io/feature_lists.h"
#include "terraingen/noise/surface_noise.h"

extern "C" {

/// WriteGeoTiff (src/raster/geotiff/geotiff_write.cpp) of `bandCount` width x height float
/// rasters (row 0 first) on the GDAL-order `transform`, no-data `nodataMode` 0 none, 1 NaN, 2
/// `nodata`; the GeoKeys given as their three tags; `compression` in TiffCompression's order.
int tgref_write_geotiff(const char* path, const float* const* bands, uint32_t bandCount,
                        uint32_t width, uint32_t height, const double* transform,
                        int nodataMode, float nodata, const uint16_t* directory,
                        uint32_t directoryCount, const double* doubles, uint32_t doubleCount,
                        const char* ascii, int compression, uint32_t tileSize, int bigTiff) {
    try {
        RasterGrid grid{width, height,
                        GeoTransform{transform[0], transform[1], transform[2], transform[3],
                                     transform[4], transform[5]}};
        std::vector<Raster<float>> rasters;
        for (uint32_t b = 0; b < bandCount; ++b) {
            Raster<float> r(grid);
            for (uint32_t row = 0; row < height; ++row) {
                for (uint32_t col = 0; col < width; ++col) {
                    r(col, row) = bands[b][size_t(row) * width + col];
                }
            }
            if (nodataMode == 1) {
                r.SetNoData(std::numeric_limits<float>::quiet_NaN());
            } else if (nodataMode == 2) {
                r.SetNoData(nodata);
            }
            rasters.push_back(std::move(r));
        }
        GeoKeys keys;
        keys.directory.assign(directory, directory + directoryCount);
        keys.doubleParams.assign(doubles, doubles + doubleCount);
        keys.asciiParams = ascii != nullptr ? ascii : "";
        GeoTiffWriteOptions options;
        options.compression = static_cast<TiffCompression>(compression);
        options.tileSize = tileSize;
        options.bigTiff = bigTiff != 0;
        if (bandCount == 1) {
            WriteGeoTiff(path, rasters.front(), keys, options);
        } else {
            WriteGeoTiff(path, rasters, keys, options);
        }
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// SyntheticSource::NoiseAt on a sphere: elevation + FractalStackAt (src/noise/surface_noise.cpp)
/// at each cell center of a width x height grid in degrees (GDAL-order `transform`).
int tgref_body_noise(const void* fractals, uint32_t count, float elevation, double radius,
                     uint32_t width, uint32_t height, const double* transform, float* out) {
    try {
        const Surface surface = Surface::Sphere(radius);
        std::vector<Fractal> stack(static_cast<const Fractal*>(fractals),
                                   static_cast<const Fractal*>(fractals) + count);
        const GeoTransform t = GeoTransform::FromGdal(
            {transform[0], transform[1], transform[2], transform[3], transform[4], transform[5]});
        for (uint32_t row = 0; row < height; ++row) {
            for (uint32_t col = 0; col < width; ++col) {
                const Vec2d p = t.PixelToWorld(double(col) + 0.5, double(row) + 0.5);
                out[size_t(row) * width + col] =
                    elevation + FractalStackAt(stack, {}, surface, p.x, p.y);
            }
        }
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// WriteCraterList (src/io/feature_lists.cpp:395) of n craters given column by column, without
/// attributes; `json` picks ListFormat::Json over Csv.
int tgref_write_crater_list(const char* path, const double* x, const double* y,
                            const double* diameter, const double* age, const uint64_t* id,
                            const uint8_t* manual, const uint8_t* replace, size_t n, int json) {
    try {
        CraterList list;
        for (size_t i = 0; i < n; ++i) {
            Crater c;
            c.x = x[i];
            c.y = y[i];
            c.diameter = diameter[i];
            c.ageGyr = age[i];
            c.id = id[i];
            c.manual = manual[i] != 0;
            c.replace = replace[i] != 0;
            list.Append(c);
        }
        WriteCraterList(list, path, json ? ListFormat::Json : ListFormat::Csv, {});
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

/// WriteBoulderList (src/io/feature_lists.cpp:412) of n boulders given column by column.
/// `values` holds 11 columns of n doubles each: x, y, diameter, height, burial, yaw, lean, tilt,
/// tiltAzimuth, wear and ground (radians for the angles); `known` marks the grounds that are set.
int tgref_write_boulder_list(const char* path, const double* values, const uint8_t* known,
                             const uint64_t* id, const uint64_t* parent, const uint32_t* piece,
                             const uint8_t* rest, const uint8_t* model, size_t n, int json) {
    try {
        BoulderList list;
        for (size_t i = 0; i < n; ++i) {
            const auto col = [&](int k) { return values[size_t(k) * n + i]; };
            Boulder b;
            b.x = col(0);
            b.y = col(1);
            b.diameter = col(2);
            b.height = col(3);
            b.burial = col(4);
            b.yaw = col(5);
            b.lean = col(6);
            b.tilt = col(7);
            b.tiltAzimuth = col(8);
            b.wear = col(9);
            if (known[i] != 0) {
                b.ground = col(10);
            }
            b.id = id[i];
            b.parent = parent[i];
            b.piece = piece[i];
            b.rest = static_cast<BoulderRest>(rest[i]);
            b.model = model[i] != 0;
            list.Append(b);
        }
        WriteBoulderList(list, path, json ? ListFormat::Json : ListFormat::Csv);
        return 0;
    } catch (const std::exception& error) {
        g_error = error.what();
        return -1;
    }
}

}  // extern "C"

#ifdef TGREF_CAPTURE
// --- capture stubs for the tg_* C ABI the adapter calls ------------------------------------
#include "tgb200.h"

namespace {

struct Capture {
    int kind = 0;  // 1 noise layer rows, 2 crater lists
    std::vector<std::vector<unsigned char>> fields;
    uint32_t width = 0, rows = 0, firstRow = 0;
    tg_nodata nodata{};
};

std::vector<Capture> g_captures;

template <typename T> std::vector<unsigned char> Bytes(const T* p, size_t count) {
    const auto* b = reinterpret_cast<const unsigned char*>(p);
    return std::vector<unsigned char>(b, b + count * sizeof(T));
}

}  // namespace

struct tg_device {
    int unused;
};

extern "C" {

int tg_open(int, tg_device** device) {
    static tg_device one{};
    *device = &one;
    return TG_OK;
}
void tg_close(tg_device*) {}
const char* tg_last_error(void) {
    return "";
}
int tg_device_name(tg_device*, char* name, size_t capacity) {
    std::snprintf(name, capacity, "capture");
    return TG_OK;
}

int tg_noise_layer_rows(tg_device*, const void* kernel, size_t kernelBytes, const float* xs,
                        const float* ys, uint32_t width, uint32_t rows, float* heights,
                        tg_nodata nodata, int, void*) {
    Capture c;
    c.kind = 1;
    c.fields = {Bytes(static_cast<const unsigned char*>(kernel), kernelBytes), Bytes(xs, width),
                Bytes(ys, rows), Bytes(heights, size_t(width) * rows)};
    c.width = width;
    c.rows = rows;
    c.nodata = nodata;
    g_captures.push_back(std::move(c));
    return TG_OK;
}

int tg_craters_apply_lists(tg_device*, const void* kernel, size_t kernelBytes, const void* records,
                           uint32_t n, const float* data, uint32_t nData, const uint32_t* heads,
                           uint32_t nHeads, const uint32_t* entries, uint32_t nEntries,
                           const float* xs, const float* xLows, const float* ys,
                           const float* yLows, uint32_t width, uint32_t rows, uint32_t firstRow,
                           float* heights, tg_nodata nodata, int, void*) {
    Capture c;
    c.kind = 2;
    c.fields = {Bytes(static_cast<const unsigned char*>(kernel), kernelBytes),
                Bytes(static_cast<const unsigned char*>(records), size_t(n) * 144),
                Bytes(data, nData),
                Bytes(heads, nHeads),
                Bytes(entries, nEntries),
                Bytes(xs, width),
                Bytes(xLows, width),
                Bytes(ys, rows),
                Bytes(yLows, size_t(firstRow) + rows),
                Bytes(heights, size_t(width) * rows)};
    c.width = width;
    c.rows = rows;
    c.firstRow = firstRow;
    c.nodata = nodata;
    g_captures.push_back(std::move(c));
    return TG_OK;
}

int tg_craters_apply_body(tg_device*, const void* kernel, size_t kernelBytes, const void* records,
                          uint32_t n, const float* data, uint32_t nData, const void* frames,
                          const uint32_t* heads, uint32_t nHeads, const uint32_t* entries,
                          uint32_t nEntries, const void* points, uint32_t width, uint32_t rows,
                          uint32_t firstRow, float* heights, tg_nodata nodata, int, void*) {
    Capture c;
    c.kind = 4;
    c.fields = {Bytes(static_cast<const unsigned char*>(kernel), kernelBytes),
                Bytes(static_cast<const unsigned char*>(records), size_t(n) * 144),
                Bytes(data, nData),
                Bytes(heads, nHeads),
                Bytes(entries, nEntries),
                Bytes(static_cast<const unsigned char*>(frames), size_t(n) * 52),
                Bytes(static_cast<const unsigned char*>(points), size_t(width) * rows * 24),
                Bytes(heights, size_t(width) * rows)};
    c.width = width;
    c.rows = rows;
    c.firstRow = firstRow;
    c.nodata = nodata;
    g_captures.push_back(std::move(c));
    return TG_OK;
}

int tg_crater_body_datums(tg_device*, const void* kernel, size_t kernelBytes,
                          const void* records, uint32_t nRecords, const float* data,
                          uint32_t nData, const void* frames, const float* bounds,
                          const uint32_t* lists, uint32_t nLists, const uint32_t* entries,
                          uint32_t nEntries, const void* positions, uint32_t width, uint32_t rows,
                          uint32_t firstRow, float* heights, tg_nodata nodata, int, void*) {
    Capture c;
    c.kind = 5;
    c.fields = {Bytes(static_cast<const unsigned char*>(kernel), kernelBytes),
                Bytes(static_cast<const unsigned char*>(records), size_t(nRecords) * 144),
                Bytes(data, nData),
                Bytes(static_cast<const unsigned char*>(frames), size_t(nRecords) * 52),
                Bytes(bounds, nRecords),
                Bytes(lists, nLists),
                Bytes(entries, nEntries),
                Bytes(static_cast<const unsigned char*>(positions), size_t(width) * rows * 24),
                Bytes(heights, size_t(width) * rows)};
    c.width = width;
    c.rows = rows;
    c.firstRow = firstRow;
    c.nodata = nodata;
    g_captures.push_back(std::move(c));
    return TG_OK;
}

int tg_crater_datums(tg_device*, const void* kernel, size_t kernelBytes, const void* records,
                     uint32_t nRecords, const float* data, uint32_t nData,
                     const float* bandFloats, uint32_t nBandFloats, const uint32_t* bandCells,
                     uint32_t nBandCells, const uint32_t* cells, uint32_t nCells,
                     const uint32_t* entries, uint32_t nEntries, const uint32_t* targets,
                     uint32_t nTargets, uint32_t width, uint32_t rows, uint32_t firstRow,
                     float* heights, int, void*) {
    Capture c;
    c.kind = 3;
    c.fields = {Bytes(static_cast<const unsigned char*>(kernel), kernelBytes),
                Bytes(static_cast<const unsigned char*>(records), size_t(nRecords) * 144),
                Bytes(data, nData),
                Bytes(bandFloats, nBandFloats),
                Bytes(bandCells, nBandCells),
                Bytes(cells, nCells),
                Bytes(entries, nEntries),
                Bytes(targets, nTargets),
                Bytes(heights, size_t(width) * rows)};
    c.width = width;
    c.rows = rows;
    c.firstRow = firstRow;
    g_captures.push_back(std::move(c));
    return TG_OK;
}

/// Captured calls so far.
int tgref_capture_count() {
    return static_cast<int>(g_captures.size());
}
void tgref_capture_clear() {
    g_captures.clear();
}
/// Call `call`'s kind, strip geometry and nodata marking.
int tgref_capture_info(int call, uint32_t* info) {
    const Capture& c = g_captures.at(static_cast<size_t>(call));
    info[0] = static_cast<uint32_t>(c.kind);
    info[1] = c.width;
    info[2] = c.rows;
    info[3] = c.firstRow;
    info[4] = c.nodata.mode;
    std::memcpy(info + 5, &c.nodata.value, sizeof(float));
    info[6] = static_cast<uint32_t>(c.fields.size());
    return 0;
}
/// Field `field` of call `call`: its bytes and size.
int tgref_capture_field(int call, int field, const void** data, size_t* bytes) {
    const Capture& c = g_captures.at(static_cast<size_t>(call));
    const auto& f = c.fields.at(static_cast<size_t>(field));
    *data = f.data();
    *bytes = f.size();
    return 0;
}

}  // extern "C"
#endif
