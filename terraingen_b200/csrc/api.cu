// The C ABI of libtgb200.so (include/tgb200.h): argument checks, device memory, host<->device
// staging and kernel launches. Kernels live in noise.cu and craters.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "kernels.h"

using namespace tgb;

namespace tgb {
namespace api {

thread_local std::string g_error;

int fail(int status, const char* format, ...) {
    char buffer[512];
    va_list args;
    va_start(args, format);
    std::vsnprintf(buffer, sizeof(buffer), format, args);
    va_end(args);
    g_error = buffer;
    return status;
}

int cuda_fail(cudaError_t err, const char* what) {
    return fail(TG_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(err));
}

int check_device(tg_device* d) {
    if (d == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "device is null");
    }
    const cudaError_t err = cudaSetDevice(d->ordinal);
    if (err != cudaSuccess) {
        return cuda_fail(err, "cudaSetDevice");
    }
    return TG_OK;
}

int check_memory(int memory) {
    if (memory != TG_MEMORY_HOST && memory != TG_MEMORY_DEVICE) {
        return fail(TG_ERROR_ARGUMENT, "memory must be TG_MEMORY_HOST or TG_MEMORY_DEVICE");
    }
    return TG_OK;
}

int to_grid(const tg_grid* g, Grid& out) {
    if (g == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "grid is null");
    }
    if (g->row_rotation != 0.0 || g->col_rotation != 0.0) {
        return fail(TG_ERROR_UNSUPPORTED, "rotated grids are not supported");
    }
    if (!(g->pixel_width != 0.0) || !(g->pixel_height != 0.0) || !std::isfinite(g->origin_x) ||
        !std::isfinite(g->origin_y) || !std::isfinite(g->pixel_width) ||
        !std::isfinite(g->pixel_height)) {
        return fail(TG_ERROR_ARGUMENT, "grid transform must be finite and invertible");
    }
    // Tile indices are kept in 16 bits (BinEntry); 65535 tiles of 16 cells bound a side, as
    // RunKernel's 65535 workgroups of 16 do (src/gpu/kernel.cpp:25).
    if (g->width > 65535u * 16u || g->height > 65535u * 16u) {
        return fail(TG_ERROR_UNSUPPORTED, "grid side above %u cells", 65535u * 16u);
    }
    out = Grid{g->width,       g->height,       g->origin_x,    g->pixel_width,
               g->row_rotation, g->origin_y,    g->col_rotation, g->pixel_height};
    return TG_OK;
}

}  // namespace api
}  // namespace tgb

using namespace tgb::api;

namespace {

NoData to_nodata(tg_nodata n) {
    return NoData{n.mode, n.value};
}

int check_nodata(tg_nodata n) {
    if (n.mode > 2u) {
        return fail(TG_ERROR_ARGUMENT, "nodata mode must be 0, 1 or 2");
    }
    return TG_OK;
}

// A buffer the kernels read: the caller's pointer in device mode, else a copy in `slot`.
// A device buffer must be aligned to `align` bytes (16 for CraterRecords, read as 16-byte words;
// 8 for doubles); a host buffer is copied into an aligned slot.
int stage_in(tg_device* d, int memory, Slot slot, const void* src, size_t bytes,
             const void** out, size_t align = sizeof(float), cudaStream_t on = nullptr) {
    if (bytes == 0) {
        *out = nullptr;
        return TG_OK;
    }
    if (src == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "a required buffer is null");
    }
    if (memory == TG_MEMORY_DEVICE) {
        if (reinterpret_cast<uintptr_t>(src) % align != 0) {
            return fail(TG_ERROR_ARGUMENT, "a device buffer is not %zu-byte aligned", align);
        }
        *out = src;
        return TG_OK;
    }
    TG_CUDA(d->slots[slot].reserve(bytes), "device allocation");
    TG_CUDA(cudaMemcpyAsync(d->slots[slot].ptr, src, bytes, cudaMemcpyHostToDevice,
                            on != nullptr ? on : d->stream),
            "copy to device");
    *out = d->slots[slot].ptr;
    return TG_OK;
}

cudaStream_t stream_of(tg_device* d, int memory, void* stream) {
    if (memory == TG_MEMORY_DEVICE && stream != nullptr) {
        return static_cast<cudaStream_t>(stream);
    }
    return d->stream;
}

template <typename T>
T* slot_ptr(tg_device* d, Slot s) {
    return static_cast<T*>(d->slots[s].ptr);
}

int copy_heights_back(tg_device* d, int memory, float* heights, const float* device,
                      size_t count) {
    if (memory != TG_MEMORY_HOST || count == 0) {
        return TG_OK;
    }
    TG_CUDA(cudaMemcpyAsync(heights, device, count * sizeof(float), cudaMemcpyDeviceToHost,
                            d->stream),
            "copy to host");
    TG_CUDA(cudaStreamSynchronize(d->stream), "synchronize");
    return TG_OK;
}

int noise_run(tg_device* d, const FractalStack& stack, const Grid& grid, const Positions& at,
              bool fill, float elevation, tg_nodata nodata, float* heights, int memory,
              void* stream) {
    const size_t cells = size_t(grid.width) * grid.height;
    if (cells == 0) {
        return TG_OK;
    }
    const cudaStream_t s = stream_of(d, memory, stream);
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
        if (!fill) {
            TG_CUDA(cudaMemcpyAsync(dh, heights, cells * sizeof(float), cudaMemcpyHostToDevice, s),
                    "copy to device");
        }
    }
    TG_CUDA(launch_noise(stack, grid, at, fill, elevation, to_nodata(nodata), dh, s),
            "noise kernel launch");
    return copy_heights_back(d, memory, heights, dh, cells);
}

int check_stack(const FractalStack& stack) {
    if (stack.count > kMaxFractals) {
        return fail(TG_ERROR_ARGUMENT, "a fractal stack holds at most %u fractals", kMaxFractals);
    }
    for (uint32_t i = 0; i < stack.count; ++i) {
        const Fractal& f = stack.fractals[i];
        if (!f.enabled) {
            continue;
        }
        // ValidateFractalParams (src/noise/validate.cpp) bounds; kernels assume them.
        if (f.octaves < 1 || f.octaves > 32 || !(f.wavelength > 0.0f) ||
            !(f.lacunarity > 1.0f) || !(f.gain > 0.0f) || f.basis > 6u || f.type > 3u ||
            f.blend > 3u) {
            return fail(TG_ERROR_ARGUMENT, "fractal %u is invalid", i);
        }
    }
    return TG_OK;
}

}  // namespace

extern "C" {

const char* tg_last_error(void) {
    return g_error.c_str();
}

int tg_open(int ordinal, tg_device** device) {
    if (device == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "device is null");
    }
    *device = nullptr;
    int count = 0;
    TG_CUDA(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (ordinal < 0 || ordinal >= count) {
        return fail(TG_ERROR_ARGUMENT, "device %d of %d", ordinal, count);
    }
    cudaDeviceProp prop;
    TG_CUDA(cudaGetDeviceProperties(&prop, ordinal), "cudaGetDeviceProperties");
    if (prop.major != 10) {
        return fail(TG_ERROR_UNSUPPORTED, "%s is sm_%d%d; this build runs on sm_100 (B200)",
                    prop.name, prop.major, prop.minor);
    }
    TG_CUDA(cudaSetDevice(ordinal), "cudaSetDevice");
    tg_device* d = new tg_device();
    d->ordinal = ordinal;
    d->name = prop.name;
    cudaError_t err = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) {
        err = cudaMallocHost(&d->pinnedStatus, 16 * sizeof(uint32_t));
    }
    if (err == cudaSuccess) {
        err = cudaStreamCreateWithFlags(&d->copyStream, cudaStreamNonBlocking);
    }
    if (err == cudaSuccess) {
        err = cudaEventCreateWithFlags(&d->copied, cudaEventDisableTiming);
    }
    for (cudaEvent_t& e : d->strips) {
        if (err == cudaSuccess) {
            err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        }
    }
    if (err != cudaSuccess) {
        delete d;
        return cuda_fail(err, "device set-up");
    }
    *device = d;
    return TG_OK;
}

void tg_close(tg_device* d) {
    if (d == nullptr) {
        return;
    }
    cudaSetDevice(d->ordinal);
    cudaStreamSynchronize(d->stream);
    for (Buffer& b : d->slots) {
        b.release();
    }
    if (d->releaseSeams != nullptr) {
        d->releaseSeams(d->seams);
    }
    if (d->pinnedStatus != nullptr) {
        cudaFreeHost(d->pinnedStatus);
    }
    if (d->recordStage != nullptr) {
        cudaFreeHost(d->recordStage);
    }
    if (d->copyStream != nullptr) {
        cudaStreamSynchronize(d->copyStream);
        cudaStreamDestroy(d->copyStream);
    }
    if (d->copied != nullptr) {
        cudaEventDestroy(d->copied);
    }
    for (cudaEvent_t e : d->strips) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    cudaStreamDestroy(d->stream);
    delete d;
}

int tg_device_name(tg_device* d, char* name, size_t capacity) {
    if (d == nullptr || name == nullptr || capacity == 0) {
        return fail(TG_ERROR_ARGUMENT, "device, name and capacity are required");
    }
    std::snprintf(name, capacity, "%s", d->name.c_str());
    return TG_OK;
}

int tg_set_wait_limit(tg_device* d, uint32_t polls) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    d->waitPolls = polls;
    return TG_OK;
}

int tg_synchronize(tg_device* d) {
    if (int s = check_device(d)) {
        return s;
    }
    TG_CUDA(cudaStreamSynchronize(d->stream), "synchronize");
    return TG_OK;
}

int tg_noise_layer(tg_device* d, const void* kernel, size_t kernel_bytes, const tg_grid* grid,
                   double origin_x, double origin_y, float* heights, tg_nodata nodata,
                   int memory, void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (kernel == nullptr || kernel_bytes != sizeof(FractalStack)) {
        return fail(TG_ERROR_ARGUMENT, "NoiseLayerKernel is %zu bytes", sizeof(FractalStack));
    }
    Grid g;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (int s = check_nodata(nodata)) {
        return s;
    }
    FractalStack stack;
    std::memcpy(&stack, kernel, sizeof(stack));
    if (int s = check_stack(stack)) {
        return s;
    }
    if (heights == nullptr && size_t(g.width) * g.height > 0) {
        return fail(TG_ERROR_ARGUMENT, "heights is null");
    }
    const Positions at{origin_x, origin_y, nullptr, nullptr};
    return noise_run(d, stack, g, at, false, 0.0f, nodata, heights, memory, stream);
}

int tg_noise_layer_rows(tg_device* d, const void* kernel, size_t kernel_bytes, const float* xs,
                        const float* ys, uint32_t width, uint32_t rows, float* heights,
                        tg_nodata nodata, int memory, void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (kernel == nullptr || kernel_bytes != sizeof(FractalStack)) {
        return fail(TG_ERROR_ARGUMENT, "NoiseLayerKernel is %zu bytes", sizeof(FractalStack));
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (int s = check_nodata(nodata)) {
        return s;
    }
    FractalStack stack;
    std::memcpy(&stack, kernel, sizeof(stack));
    if (int s = check_stack(stack)) {
        return s;
    }
    if (size_t(width) * rows == 0) {
        return TG_OK;
    }
    if (heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "heights is null");
    }
    const void* dxs = nullptr;
    const void* dys = nullptr;
    if (int s = stage_in(d, memory, kXs, xs, width * sizeof(float), &dxs)) {
        return s;
    }
    if (int s = stage_in(d, memory, kYs, ys, rows * sizeof(float), &dys)) {
        return s;
    }
    // Unit transform: the positions come from xs / ys.
    const Grid g{width, rows, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};
    const Positions at{0.0, 0.0, static_cast<const float*>(dxs), static_cast<const float*>(dys)};
    return noise_run(d, stack, g, at, false, 0.0f, nodata, heights, memory, stream);
}

int tg_noise_source(tg_device* d, const void* fractals, uint32_t count, float elevation,
                    const tg_grid* grid, float* heights, int memory, void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (count > kMaxFractals || (count > 0 && fractals == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "at most %u fractals, and a pointer to them",
                    kMaxFractals);
    }
    Grid g;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    FractalStack stack;
    std::memset(&stack, 0, sizeof(stack));
    std::memcpy(stack.fractals, fractals, count * sizeof(Fractal));
    stack.count = count;
    if (int s = check_stack(stack)) {
        return s;
    }
    if (heights == nullptr && size_t(g.width) * g.height > 0) {
        return fail(TG_ERROR_ARGUMENT, "heights is null");
    }
    // SyntheticSource evaluates at float(world x), its origin being zero
    // (synthetic_source.cpp:76-80, surface_noise.cpp:31-33).
    const Positions at{0.0, 0.0, nullptr, nullptr};
    return noise_run(d, stack, g, at, true, elevation, tg_nodata{0u, 0.0f}, heights, memory,
                     stream);
}

int tg_noise_source_body(tg_device* d, const void* fractals, uint32_t count, float elevation,
                         const tg_grid* grid, double radius, float* heights, int memory,
                         void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (count > kMaxFractals || (count > 0 && fractals == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "at most %u fractals, and a pointer to them",
                    kMaxFractals);
    }
    if (!(radius > 0.0) || !std::isfinite(radius)) {
        return fail(TG_ERROR_ARGUMENT, "a sphere's radius must be positive and finite");
    }
    Grid g;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    FractalStack stack;
    std::memset(&stack, 0, sizeof(stack));
    std::memcpy(stack.fractals, fractals, count * sizeof(Fractal));
    stack.count = count;
    if (int s = check_stack(stack)) {
        return s;
    }
    const size_t cells = size_t(g.width) * g.height;
    if (cells == 0) {
        return TG_OK;
    }
    if (heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "heights is null");
    }
    // Cell centers in degrees as Raster::CellCenter gives them (GeoTransform::PixelToWorld, the
    // rotation terms 0), their cosines and sines with the host's libm as the reference's
    // UnitVector takes them (surface.cpp:45-50).
    constexpr double kPi = 3.141592653589793238462643383279502884;
    constexpr double kDegree = kPi / 180.0;
    std::vector<double> trig(2 * size_t(g.width) + 2 * size_t(g.height));
    for (uint32_t col = 0; col < g.width; ++col) {
        const double lon = (g.originX + (double(col) + 0.5) * g.pixelWidth + 0.5 * g.rowRotation) *
                           kDegree;
        trig[2 * col] = std::cos(lon);
        trig[2 * col + 1] = std::sin(lon);
    }
    double* latTrig = trig.data() + 2 * size_t(g.width);
    for (uint32_t row = 0; row < g.height; ++row) {
        const double lat =
            (g.originY + 0.5 * g.colRotation + (double(row) + 0.5) * g.pixelHeight) * kDegree;
        latTrig[2 * row] = std::cos(lat);
        latTrig[2 * row + 1] = std::sin(lat);
    }
    const cudaStream_t s = stream_of(d, memory, stream);
    const void* dtrig = nullptr;
    if (int st = stage_in(d, TG_MEMORY_HOST, kProbeIn, trig.data(), trig.size() * sizeof(double),
                          &dtrig)) {
        return st;
    }
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
    }
    const double* dl = static_cast<const double*>(dtrig);
    TG_CUDA(launch_noise_body(stack, elevation, g.width, g.height, dl, dl + 2 * size_t(g.width),
                              radius, dh, s),
            "body noise launch");
    return copy_heights_back(d, memory, heights, dh, cells);
}

int tg_noise_probe(tg_device* d, const float* xy, uint32_t n, uint32_t seed, uint32_t* hashes,
                   float* values, int memory) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int s = check_memory(memory)) {
        return s;
    }
    if (n == 0) {
        return TG_OK;
    }
    if (xy == nullptr || hashes == nullptr || values == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "probe buffers are required");
    }
    const void* dxy = nullptr;
    if (int s = stage_in(d, memory, kProbeIn, xy, size_t(n) * 2 * sizeof(float), &dxy)) {
        return s;
    }
    uint32_t* dh = hashes;
    float* dv = values;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kProbeHashes].reserve(size_t(n) * 4 * sizeof(uint32_t)), "allocation");
        TG_CUDA(d->slots[kProbeValues].reserve(size_t(n) * 12 * sizeof(float)), "allocation");
        dh = slot_ptr<uint32_t>(d, kProbeHashes);
        dv = slot_ptr<float>(d, kProbeValues);
    }
    TG_CUDA(launch_noise_probe(static_cast<const float*>(dxy), n, seed, dh, dv, d->stream),
            "probe launch");
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(cudaMemcpyAsync(hashes, dh, size_t(n) * 4 * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, d->stream),
                "copy to host");
        TG_CUDA(cudaMemcpyAsync(values, dv, size_t(n) * 12 * sizeof(float), cudaMemcpyDeviceToHost,
                                d->stream),
                "copy to host");
    }
    TG_CUDA(cudaStreamSynchronize(d->stream), "synchronize");
    return TG_OK;
}

}  // extern "C"

namespace {

// The crater pipeline's binning on stream `s` (footprints, count, scan, lean craters, scatter):
// what the shaping launches need, with no round trip to the host. The entries get the capacity
// the device's slot already has (at least a guess from the craters and bins); when the scan's
// total is larger the scatter and the shaping do nothing (crater_bins_usable) and layers_settle
// grows the slot and asks for the layer again. `any` is false when no cell can need a crater.
struct CraterPrep {
    CraterBins bins{};
    const void* leans = nullptr;  // the lean craters (plain kernel options), else null
    bool extras = false;          // launch the extras pass (it returns at once without work)
    bool any = false;
    size_t entryBytes = 0;
};

int crater_prepare(tg_device* d, const CraterShapeKernel& k, const CraterRecord* rec, uint32_t n,
                   const float* data, uint32_t nData, const double* foot, const Grid& g,
                   cudaStream_t s, CraterPrep& p) {
    p = CraterPrep{};
    if (size_t(g.width) * g.height == 0 || n == 0) {
        return TG_OK;
    }
    CraterBins& bins = p.bins;
    bins.binsX = (g.width + kBinCells - 1) / kBinCells;
    bins.binsY = (g.height + kBinCells - 1) / kBinCells;
    const uint32_t nbins = bins.binsX * bins.binsY;
    TG_CUDA(d->slots[kCounts].reserve((size_t(nbins) + 1) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kCursor].reserve(size_t(nbins) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kBoxes].reserve(size_t(n) * sizeof(int4)), "allocation");
    TG_CUDA(d->slots[kCulls].reserve(size_t(n) * sizeof(float)), "allocation");
    TG_CUDA(d->slots[kScan].reserve(scan_scratch_words(std::max(nbins, n)) * sizeof(uint32_t)),
            "allocation");
    TG_CUDA(d->slots[kStatus].reserve(4 * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kPairStart].reserve((size_t(n) + 1) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kExtrasMark].reserve(size_t(nbins) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kExtrasList].reserve((size_t(nbins) + 1) * sizeof(uint32_t)), "allocation");
    bins.counts = slot_ptr<uint32_t>(d, kCounts);
    bins.cursor = slot_ptr<uint32_t>(d, kCursor);
    bins.boxes = slot_ptr<int4>(d, kBoxes);
    bins.culls = slot_ptr<float>(d, kCulls);
    bins.total = slot_ptr<uint32_t>(d, kStatus);
    bins.pairStart = slot_ptr<uint32_t>(d, kPairStart);
    bins.extrasMark = slot_ptr<uint32_t>(d, kExtrasMark);
    bins.extrasList = slot_ptr<uint32_t>(d, kExtrasList);
    TG_CUDA(cudaMemsetAsync(bins.counts, 0, (size_t(nbins) + 1) * sizeof(uint32_t), s), "memset");
    TG_CUDA(cudaMemsetAsync(bins.cursor, 0, size_t(nbins) * sizeof(uint32_t), s), "memset");
    TG_CUDA(cudaMemsetAsync(bins.total, 0, 4 * sizeof(uint32_t), s), "memset");
    TG_CUDA(cudaMemsetAsync(bins.extrasMark, 0, size_t(nbins) * sizeof(uint32_t), s), "memset");
    TG_CUDA(cudaMemsetAsync(bins.extrasList, 0, sizeof(uint32_t), s), "memset");
    TG_CUDA(launch_crater_count(k, rec, n, data, foot, g, bins, slot_ptr<uint32_t>(d, kScan), s),
            "crater count launch");
    TG_CUDA(launch_exclusive_scan(bins.counts, nbins, slot_ptr<uint32_t>(d, kScan), s),
            "scan launch");
    // The entries get the slot's capacity, at least a guess; a larger total is found on the
    // device and settled after the layer.
    const bool lean = crater_lean_entries(k);
    p.entryBytes = lean ? kLeanEntryBytes : sizeof(BinEntry);
    const size_t guess = (lean ? 4 : 2) * size_t(n) + nbins;
    const size_t have = d->slots[kBinEntries].bytes / p.entryBytes;
    TG_CUDA(d->slots[kBinEntries].reserve(std::max(have, guess) * p.entryBytes), "allocation");
    bins.entries = slot_ptr<BinEntry>(d, kBinEntries);
    bins.capacity = uint32_t(std::min<size_t>(d->slots[kBinEntries].bytes / p.entryBytes,
                                              0xffffffffu));
    if (lean) {
        TG_CUDA(d->slots[kHarmonics].reserve(size_t(n) * kLeanCraterBytes), "allocation");
        p.leans = d->slots[kHarmonics].ptr;
        TG_CUDA(launch_crater_lean(k, rec, n, data, bins, d->slots[kHarmonics].ptr, s),
                "lean crater launch");
    }
    TG_CUDA(launch_crater_scatter(k, rec, n, g, bins, p.leans, s), "crater scatter launch");
    p.extras = lean;
    p.any = true;
    return TG_OK;
}

// The words a layer's settling reads, copied after its last kernel on stream `s`: for craters
// the entries needed and the status (flags, pairs), for boulders the same at kBoulderWords.
constexpr uint32_t kCraterWords = 0, kBoulderWords = 8;  // of tg_device::pinnedStatus's 16

int crater_finish(tg_device* d, const CraterPrep& p, cudaStream_t s) {
    if (!p.any) {
        return TG_OK;
    }
    const uint32_t nbins = p.bins.binsX * p.bins.binsY;
    TG_CUDA(cudaMemcpyAsync(d->pinnedStatus + kCraterWords, p.bins.counts + nbins,
                            sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy to host");
    TG_CUDA(cudaMemcpyAsync(d->pinnedStatus + kCraterWords + 1, p.bins.total + 1,
                            3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy to host");
    return TG_OK;
}

// The boulder pipeline's binning on stream `s` (count, scan, scatter), its counts, cursor and
// status in the given slots, sized as the craters' are (no round trip to the host; see
// CraterPrep). `any` is false when no cell can need a boulder.
struct BoulderPrep {
    BoulderBins bins{};
    uint32_t* status = nullptr;
    bool any = false;
};

int boulder_prepare(tg_device* d, const BoulderRecord* rec, uint32_t n, double width,
                    const Grid& g, cudaStream_t s, Slot countSlot, Slot cursorSlot,
                    Slot statusSlot, BoulderPrep& p) {
    p = BoulderPrep{};
    if (size_t(g.width) * g.height == 0 || n == 0) {
        return TG_OK;
    }
    BoulderBins& bins = p.bins;
    bins.binsX = (g.width + kBinCells - 1) / kBinCells;
    bins.binsY = (g.height + kBinCells - 1) / kBinCells;
    const uint32_t nbins = bins.binsX * bins.binsY;
    TG_CUDA(d->slots[countSlot].reserve((size_t(nbins) + 1) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[cursorSlot].reserve(size_t(nbins) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kBoulderWindows].reserve(size_t(n) * sizeof(int4)), "allocation");
    TG_CUDA(d->slots[kScan].reserve(scan_scratch_words(nbins) * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[statusSlot].reserve(4 * sizeof(uint32_t)), "allocation");
    const size_t guess = 2 * size_t(n) + nbins;
    const size_t have = d->slots[kBoulderEntries].bytes / sizeof(BoulderEntry);
    TG_CUDA(d->slots[kBoulderEntries].reserve(std::max(have, guess) * sizeof(BoulderEntry)),
            "allocation");
    bins.counts = slot_ptr<uint32_t>(d, countSlot);
    bins.cursor = slot_ptr<uint32_t>(d, cursorSlot);
    bins.windows = slot_ptr<int4>(d, kBoulderWindows);
    bins.entries = slot_ptr<BoulderEntry>(d, kBoulderEntries);
    bins.capacity = uint32_t(std::min<size_t>(
        d->slots[kBoulderEntries].bytes / sizeof(BoulderEntry), 0xffffffffu));
    p.status = slot_ptr<uint32_t>(d, statusSlot);
    TG_CUDA(cudaMemsetAsync(bins.counts, 0, (size_t(nbins) + 1) * sizeof(uint32_t), s), "memset");
    TG_CUDA(cudaMemsetAsync(bins.cursor, 0, size_t(nbins) * sizeof(uint32_t), s), "memset");
    TG_CUDA(cudaMemsetAsync(p.status, 0, 4 * sizeof(uint32_t), s), "memset");
    TG_CUDA(launch_boulder_count(rec, n, g, width, bins, s), "boulder count launch");
    TG_CUDA(launch_exclusive_scan(bins.counts, nbins, slot_ptr<uint32_t>(d, kScan), s),
            "scan launch");
    TG_CUDA(launch_boulder_scatter(rec, n, bins, s), "boulder scatter launch");
    p.any = true;
    return TG_OK;
}

int boulder_finish(tg_device* d, const BoulderPrep& p, cudaStream_t s) {
    if (!p.any) {
        return TG_OK;
    }
    const uint32_t nbins = p.bins.binsX * p.bins.binsY;
    TG_CUDA(cudaMemcpyAsync(d->pinnedStatus + kBoulderWords, p.bins.counts + nbins,
                            sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy to host");
    TG_CUDA(cudaMemcpyAsync(d->pinnedStatus + kBoulderWords + 1, p.status, 4 * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, s),
            "copy to host");
    return TG_OK;
}

// After the layers' streams are synchronized: their pair counts and errors, and whether a layer's
// entries outgrew their capacity (`again`: its slot is grown to the total and the caller runs the
// layers again from the heights they started from).
int layers_settle(tg_device* d, const CraterPrep* cp, const BoulderPrep* bp, bool& again) {
    again = false;
    const uint32_t* w = d->pinnedStatus;
    if (cp != nullptr && cp->any) {
        const uint32_t needed = w[kCraterWords], flags = w[kCraterWords + 1];
        if (flags & 1u) {
            return fail(TG_ERROR_UNSUPPORTED,
                        "craters with a datum need the ordered form (tg_craters_apply_lists)");
        }
        if (needed > cp->bins.capacity) {
            TG_CUDA(d->slots[kBinEntries].reserve(size_t(needed) * cp->entryBytes), "allocation");
            again = true;
        } else {
            if (flags & 2u) {
                return fail(TG_ERROR_TIMEOUT, "a crater bin's staged copy did not arrive");
            }
            d->craterPairs = (static_cast<unsigned long long>(w[kCraterWords + 3]) << 32) |
                             w[kCraterWords + 2];
        }
    }
    if (bp != nullptr && bp->any) {
        const uint32_t needed = w[kBoulderWords];
        const uint32_t* status = w + kBoulderWords + 1;
        if (needed > bp->bins.capacity) {
            TG_CUDA(d->slots[kBoulderEntries].reserve(size_t(needed) * sizeof(BoulderEntry)),
                    "allocation");
            again = true;
        } else {
            if (status[0] & 2u) {
                return fail(TG_ERROR_TIMEOUT, "a boulder bin's staged copy did not arrive");
            }
            d->boulderPairs = (static_cast<unsigned long long>(status[3]) << 32) | status[2];
        }
    }
    return TG_OK;
}

// The crater layer on device heights `dh` (stream `s`): binning, shaping and one synchronize at
// the end; again once with grown entries when they did not fit (the heights are untouched then).
int craters_device(tg_device* d, const CraterShapeKernel& k, const CraterRecord* rec, uint32_t n,
                   const float* data, uint32_t nData, const double* foot, const Grid& g,
                   float* dh, tg_nodata nodata, cudaStream_t s) {
    for (int attempt = 0; attempt < 2; ++attempt) {
        CraterPrep p;
        if (int st = crater_prepare(d, k, rec, n, data, nData, foot, g, s, p)) {
            return st;
        }
        if (!p.any) {
            return TG_OK;
        }
        TG_CUDA(launch_crater_shape(k, rec, data, p.leans, p.extras, g, to_nodata(nodata),
                                    p.bins, dh, s, 0, 0xffffffffu, d->waitPolls),
                "crater shape launch");
        if (int st = crater_finish(d, p, s)) {
            return st;
        }
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        bool again = false;
        if (int st = layers_settle(d, &p, nullptr, again)) {
            return st;
        }
        if (!again) {
            return TG_OK;
        }
    }
    return fail(TG_ERROR_MEMORY, "the crater entries did not fit after growing");
}

// The boulder pipeline on device heights (count, scan, scatter, bake), as craters_device.
int boulders_device(tg_device* d, const BoulderRecord* rec, uint32_t n, double width,
                    const Grid& g, float* dh, tg_nodata nodata, cudaStream_t s) {
    for (int attempt = 0; attempt < 2; ++attempt) {
        BoulderPrep p;
        if (int st = boulder_prepare(d, rec, n, width, g, s, kCounts, kCursor, kStatus, p)) {
            return st;
        }
        if (!p.any) {
            return TG_OK;
        }
        TG_CUDA(launch_boulder_bake(g, width, to_nodata(nodata), p.bins, dh, p.status, s, 0,
                                    0xffffffffu, d->waitPolls),
                "boulder bake launch");
        if (int st = boulder_finish(d, p, s)) {
            return st;
        }
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        bool again = false;
        if (int st = layers_settle(d, nullptr, &p, again)) {
            return st;
        }
        if (!again) {
            return TG_OK;
        }
    }
    return fail(TG_ERROR_MEMORY, "the boulder entries did not fit after growing");
}

int check_boulders(const void* boulders, uint32_t n) {
    const BoulderRecord* b = static_cast<const BoulderRecord*>(boulders);
    for (uint32_t i = 0; i < n; ++i) {
        if (!(b[i].diameter > 0.0) || !std::isfinite(b[i].x) || !std::isfinite(b[i].y) ||
            !(b[i].exposedHeight >= 0.0) || !(b[i].weight >= 0.0 && b[i].weight <= 1.0)) {
            return fail(TG_ERROR_ARGUMENT, "boulder %u is invalid", i);
        }
    }
    return TG_OK;
}

}  // namespace

extern "C" {

int tg_craters_apply(tg_device* d, const void* kernel, size_t kernel_bytes, const void* records,
                     uint32_t n, const float* data, uint32_t n_data, const double* footprints,
                     const tg_grid* grid, float* heights, tg_nodata nodata, int memory,
                     void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (kernel == nullptr || kernel_bytes != sizeof(CraterShapeKernel)) {
        return fail(TG_ERROR_ARGUMENT, "CraterShapeKernel is %zu bytes", sizeof(CraterShapeKernel));
    }
    Grid g;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (int s = check_nodata(nodata)) {
        return s;
    }
    const size_t cells = size_t(g.width) * g.height;
    if (cells == 0 || n == 0) {
        return TG_OK;
    }
    if (heights == nullptr || records == nullptr || (n_data > 0 && data == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "heights, records and data are required");
    }
    CraterShapeKernel k;
    std::memcpy(&k, kernel, sizeof(k));
    const cudaStream_t s = stream_of(d, memory, stream);
    const void* drec = nullptr;
    const void* ddata = nullptr;
    const void* dfoot = nullptr;
    if (int st = stage_in(d, memory, kRecords, records, size_t(n) * sizeof(CraterRecord), &drec, 16)) {
        return st;
    }
    if (int st = stage_in(d, memory, kData, data, size_t(n_data) * sizeof(float), &ddata)) {
        return st;
    }
    if (footprints != nullptr) {
        if (int st = stage_in(d, memory, kFootprints, footprints, size_t(n) * 3 * sizeof(double),
                              &dfoot, 8)) {
            return st;
        }
    }
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
        TG_CUDA(cudaMemcpyAsync(dh, heights, cells * sizeof(float), cudaMemcpyHostToDevice, s),
                "copy to device");
    }
    if (int st = craters_device(d, k, static_cast<const CraterRecord*>(drec), n,
                                static_cast<const float*>(ddata), n_data,
                                static_cast<const double*>(dfoot), g, dh, nodata, s)) {
        return st;
    }
    return copy_heights_back(d, memory, heights, dh, cells);
}

int tg_craters_apply_lists(tg_device* d, const void* kernel, size_t kernel_bytes,
                           const void* records, uint32_t n, const float* data, uint32_t n_data,
                           const uint32_t* heads, uint32_t n_heads, const uint32_t* entries,
                           uint32_t n_entries, const float* xs, const float* x_lows,
                           const float* ys, const float* y_lows, uint32_t width, uint32_t rows,
                           uint32_t first_row, float* heights, tg_nodata nodata, int memory,
                           void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (kernel == nullptr || kernel_bytes != sizeof(CraterShapeKernel)) {
        return fail(TG_ERROR_ARGUMENT, "CraterShapeKernel is %zu bytes", sizeof(CraterShapeKernel));
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (int s = check_nodata(nodata)) {
        return s;
    }
    const size_t cells = size_t(width) * rows;
    if (cells == 0) {
        return TG_OK;
    }
    if (heads == nullptr || n_heads < 3 || entries == nullptr || n_entries == 0 ||
        heights == nullptr || xs == nullptr || x_lows == nullptr || ys == nullptr ||
        y_lows == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "tile lists, positions and heights are required");
    }
    // The lists' geometry is read on the device; check it here where the host can.
    if (memory == TG_MEMORY_HOST) {
        if (heads[2] != 0u) {
            return fail(TG_ERROR_UNSUPPORTED, "crater tiles on a body are not supported");
        }
        const uint32_t tilesX = heads[0], side = heads[1];
        if (side == 0 || tilesX == 0 || tilesX < (width + side - 1) / side ||
            n_heads < 3 + 2 * tilesX * ((first_row + rows + side - 1) / side)) {
            return fail(TG_ERROR_ARGUMENT, "tile heads do not cover the strip");
        }
        for (uint32_t t = 3; t + 1 < n_heads; t += 2) {
            if (uint64_t(heads[t]) + heads[t + 1] > n_entries) {
                return fail(TG_ERROR_ARGUMENT, "tile list past the entries");
            }
        }
        for (uint32_t e = 0; e < n_entries; ++e) {
            if (entries[e] >= n && !(n == 0 && e == 0)) {
                return fail(TG_ERROR_ARGUMENT, "entry %u names crater %u of %u", e, entries[e], n);
            }
        }
    }
    CraterShapeKernel k;
    std::memcpy(&k, kernel, sizeof(k));
    const cudaStream_t s = stream_of(d, memory, stream);
    const void *drec, *ddata, *dheads, *dentries, *dxs, *dxl, *dys, *dyl;
    if (int st = stage_in(d, memory, kRecords, records, size_t(n) * sizeof(CraterRecord), &drec, 16)) {
        return st;
    }
    if (int st = stage_in(d, memory, kData, data, size_t(n_data) * sizeof(float), &ddata)) {
        return st;
    }
    if (int st = stage_in(d, memory, kHeads, heads, size_t(n_heads) * sizeof(uint32_t), &dheads)) {
        return st;
    }
    if (int st = stage_in(d, memory, kEntries, entries, size_t(n_entries) * sizeof(uint32_t),
                          &dentries)) {
        return st;
    }
    if (int st = stage_in(d, memory, kXs, xs, size_t(width) * sizeof(float), &dxs)) {
        return st;
    }
    if (int st = stage_in(d, memory, kXLows, x_lows, size_t(width) * sizeof(float), &dxl)) {
        return st;
    }
    if (int st = stage_in(d, memory, kYs, ys, size_t(rows) * sizeof(float), &dys)) {
        return st;
    }
    if (int st = stage_in(d, memory, kYLows, y_lows, size_t(first_row + rows) * sizeof(float),
                          &dyl)) {
        return st;
    }
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
        TG_CUDA(cudaMemcpyAsync(dh, heights, cells * sizeof(float), cudaMemcpyHostToDevice, s),
                "copy to device");
    }
    TG_CUDA(launch_crater_shape_lists(
                k, static_cast<const CraterRecord*>(drec), static_cast<const float*>(ddata),
                static_cast<const uint32_t*>(dheads), static_cast<const uint32_t*>(dentries), width,
                rows, first_row, static_cast<const float*>(dxs), static_cast<const float*>(dxl),
                static_cast<const float*>(dys), static_cast<const float*>(dyl), to_nodata(nodata),
                dh, s),
            "crater lists launch");
    return copy_heights_back(d, memory, heights, dh, cells);
}

int tg_craters_apply_body(tg_device* d, const void* kernel, size_t kernel_bytes,
                          const void* records, uint32_t n, const float* data, uint32_t n_data,
                          const void* frames, const uint32_t* heads, uint32_t n_heads,
                          const uint32_t* entries, uint32_t n_entries, const void* points,
                          uint32_t width, uint32_t rows, uint32_t first_row, float* heights,
                          tg_nodata nodata, int memory, void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (kernel == nullptr || kernel_bytes != sizeof(CraterShapeKernel)) {
        return fail(TG_ERROR_ARGUMENT, "CraterShapeKernel is %zu bytes", sizeof(CraterShapeKernel));
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (int s = check_nodata(nodata)) {
        return s;
    }
    const size_t cells = size_t(width) * rows;
    if (cells == 0) {
        return TG_OK;
    }
    if (heads == nullptr || n_heads < 3 || entries == nullptr || n_entries == 0 ||
        heights == nullptr || points == nullptr || (n > 0 && frames == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "tile lists, frames, points and heights are required");
    }
    if (memory == TG_MEMORY_HOST) {
        const uint32_t tilesX = heads[0], side = heads[1];
        if (side == 0 || tilesX == 0 || tilesX < (width + side - 1) / side ||
            n_heads < 3 + 2 * tilesX * ((first_row + rows + side - 1) / side)) {
            return fail(TG_ERROR_ARGUMENT, "tile heads do not cover the strip");
        }
        for (uint32_t t = 3; t + 1 < n_heads; t += 2) {
            if (uint64_t(heads[t]) + heads[t + 1] > n_entries) {
                return fail(TG_ERROR_ARGUMENT, "tile list past the entries");
            }
        }
        for (uint32_t e = 0; e < n_entries; ++e) {
            if (entries[e] >= n && !(n == 0 && e == 0)) {
                return fail(TG_ERROR_ARGUMENT, "entry %u names crater %u of %u", e, entries[e], n);
            }
        }
    }
    CraterShapeKernel k;
    std::memcpy(&k, kernel, sizeof(k));
    const cudaStream_t s = stream_of(d, memory, stream);
    const void *drec, *dframes, *ddata, *dheads, *dentries, *dpoints;
    if (int st = stage_in(d, memory, kRecords, records, size_t(n) * sizeof(CraterRecord), &drec, 16)) {
        return st;
    }
    if (int st = stage_in(d, memory, kFrames, frames, size_t(n) * sizeof(CraterFrame), &dframes)) {
        return st;
    }
    if (int st = stage_in(d, memory, kData, data, size_t(n_data) * sizeof(float), &ddata)) {
        return st;
    }
    if (int st = stage_in(d, memory, kHeads, heads, size_t(n_heads) * sizeof(uint32_t), &dheads)) {
        return st;
    }
    if (int st = stage_in(d, memory, kEntries, entries, size_t(n_entries) * sizeof(uint32_t),
                          &dentries)) {
        return st;
    }
    if (int st = stage_in(d, memory, kPoints, points, cells * sizeof(SplitPoint), &dpoints)) {
        return st;
    }
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
        TG_CUDA(cudaMemcpyAsync(dh, heights, cells * sizeof(float), cudaMemcpyHostToDevice, s),
                "copy to device");
    }
    TG_CUDA(launch_crater_shape_body(k, static_cast<const CraterRecord*>(drec),
                                     static_cast<const CraterFrame*>(dframes),
                                     static_cast<const float*>(ddata),
                                     static_cast<const uint32_t*>(dheads),
                                     static_cast<const uint32_t*>(dentries), width, rows,
                                     first_row, static_cast<const SplitPoint*>(dpoints),
                                     to_nodata(nodata), dh, s),
            "crater body launch");
    return copy_heights_back(d, memory, heights, dh, cells);
}

int tg_boulders_bake(tg_device* d, const void* boulders, uint32_t n, double width,
                     const tg_grid* grid, float* heights, tg_nodata nodata, int memory,
                     void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    Grid g;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (int s = check_nodata(nodata)) {
        return s;
    }
    if (!(width >= 0.0) || !std::isfinite(width)) {
        return fail(TG_ERROR_ARGUMENT, "the dome width must be finite and not negative");
    }
    const size_t cells = size_t(g.width) * g.height;
    if (cells == 0 || n == 0) {
        return TG_OK;
    }
    if (heights == nullptr || boulders == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "heights and boulders are required");
    }
    if (memory == TG_MEMORY_HOST) {
        if (int st = check_boulders(boulders, n)) {
            return st;
        }
    }
    const cudaStream_t s = stream_of(d, memory, stream);
    const void* db = nullptr;
    if (int st = stage_in(d, memory, kBoulders, boulders, size_t(n) * sizeof(BoulderRecord), &db, 8)) {
        return st;
    }
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
        TG_CUDA(cudaMemcpyAsync(dh, heights, cells * sizeof(float), cudaMemcpyHostToDevice, s),
                "copy to device");
    }
    if (int st = boulders_device(d, static_cast<const BoulderRecord*>(db), n, width, g, dh,
                                 nodata, s)) {
        return st;
    }
    return copy_heights_back(d, memory, heights, dh, cells);
}

int tg_evaluate(tg_device* d, const tg_terrain* t, const tg_grid* grid, float* heights,
                int memory, void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (t == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "terrain is null");
    }
    Grid g;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    const size_t cells = size_t(g.width) * g.height;
    if (cells == 0) {
        return TG_OK;
    }
    if (heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "heights is null");
    }
    if (t->n_fractals > kMaxFractals || (t->n_fractals > 0 && t->fractals == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "at most %u source fractals", kMaxFractals);
    }
    FractalStack source;
    std::memset(&source, 0, sizeof(source));
    if (t->n_fractals > 0) {
        std::memcpy(source.fractals, t->fractals, t->n_fractals * sizeof(Fractal));
    }
    source.count = t->n_fractals;
    if (int s = check_stack(source)) {
        return s;
    }
    FractalStack layer;
    if (t->noise_layer != nullptr) {
        std::memcpy(&layer, t->noise_layer, sizeof(layer));
        if (int s = check_stack(layer)) {
            return s;
        }
    }
    CraterShapeKernel k;
    if (t->n_craters > 0) {
        if (t->crater_kernel == nullptr || t->crater_records == nullptr ||
            (t->n_crater_data > 0 && t->crater_data == nullptr)) {
            return fail(TG_ERROR_ARGUMENT, "craters need a kernel, records and data");
        }
        std::memcpy(&k, t->crater_kernel, sizeof(k));
    }
    if (t->n_boulders > 0) {
        if (t->boulders == nullptr || !(t->boulder_width >= 0.0)) {
            return fail(TG_ERROR_ARGUMENT, "boulders need records and a width");
        }
        if (memory == TG_MEMORY_HOST) {
            if (int st = check_boulders(t->boulders, t->n_boulders)) {
                return st;
            }
        }
    }
    const cudaStream_t s = stream_of(d, memory, stream);
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
    }
    // Terrain::Fill: the source, then each layer in order (src/pipeline/terrain.cpp:299-331).
    const Positions origin{0.0, 0.0, nullptr, nullptr};
    auto sources = [&]() -> int {
        TG_CUDA(launch_noise(source, g, origin, true, t->elevation, NoData{0u, 0.0f}, dh, s),
                "noise source launch");
        if (t->noise_layer != nullptr) {
            TG_CUDA(launch_noise(layer, g, origin, false, 0.0f, NoData{0u, 0.0f}, dh, s),
                    "noise layer launch");
        }
        return TG_OK;
    };
    if (int st = sources()) {
        return st;
    }
    // Host-memory layer inputs are copied on the device's copy stream while the source's
    // kernels run; the layers wait for them.
    const cudaStream_t on = memory == TG_MEMORY_HOST ? d->copyStream : nullptr;
    const void *drec = nullptr, *ddata = nullptr, *dfoot = nullptr, *db = nullptr;
    if (t->n_craters > 0) {
        if (int st = stage_in(d, memory, kRecords, t->crater_records,
                              size_t(t->n_craters) * sizeof(CraterRecord), &drec, 16, on)) {
            return st;
        }
        if (int st = stage_in(d, memory, kData, t->crater_data,
                              size_t(t->n_crater_data) * sizeof(float), &ddata,
                              sizeof(float), on)) {
            return st;
        }
        if (t->crater_footprints != nullptr) {
            if (int st = stage_in(d, memory, kFootprints, t->crater_footprints,
                                  size_t(t->n_craters) * 3 * sizeof(double), &dfoot, 8, on)) {
                return st;
            }
        }
    }
    if (t->n_boulders > 0) {
        if (int st = stage_in(d, memory, kBoulders, t->boulders,
                              size_t(t->n_boulders) * sizeof(BoulderRecord), &db, 8, on)) {
            return st;
        }
    }
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(cudaEventRecord(d->copied, d->copyStream), "event");
        TG_CUDA(cudaStreamWaitEvent(s, d->copied, 0), "event wait");
    }
    const bool layers = t->n_craters > 0 || t->n_boulders > 0;
    if (!layers) {
        return copy_heights_back(d, memory, heights, dh, cells);
    }
    // The layers, then one synchronize; when a layer's binned entries outgrew their capacity the
    // kernels after its scan did nothing, and the whole evaluation runs again with grown entries.
    const NoData none{0u, 0.0f};
    auto drain = [&](int st) {
        cudaStreamSynchronize(d->copyStream);
        return st;
    };
    for (int attempt = 0; attempt < 2; ++attempt) {
        if (attempt > 0) {
            if (int st = sources()) {
                return st;
            }
        }
        CraterPrep cp;
        BoulderPrep bp;
        if (t->n_craters > 0) {
            if (int st = crater_prepare(d, k, static_cast<const CraterRecord*>(drec),
                                        t->n_craters, static_cast<const float*>(ddata),
                                        t->n_crater_data, static_cast<const double*>(dfoot), g,
                                        s, cp)) {
                return st;
            }
        }
        if (t->n_boulders > 0) {
            if (int st = boulder_prepare(d, static_cast<const BoulderRecord*>(db),
                                         t->n_boulders, t->boulder_width, g, s, kBoulderCounts,
                                         kBoulderCursor, kBoulderStatus, bp)) {
                return st;
            }
        }
        // Host memory: the layers by strips of bin rows, each strip copied out on the copy
        // stream while the next is shaped and baked. Device memory: one launch per layer.
        const uint32_t binRows = (g.height + kBinCells - 1) / kBinCells;
        const uint32_t strips = memory == TG_MEMORY_HOST ? std::min<uint32_t>(8u, binRows) : 1u;
        const uint32_t per = (binRows + strips - 1) / strips;
        for (uint32_t k0 = 0, q = 0; k0 < binRows; k0 += per, ++q) {
            const uint32_t rows = std::min(per, binRows - k0);
            if (cp.any) {
                if (cudaError_t e = launch_crater_shape(
                        k, static_cast<const CraterRecord*>(drec),
                        static_cast<const float*>(ddata), cp.leans, cp.extras, g, none, cp.bins,
                        dh, s, k0, rows, d->waitPolls)) {
                    return drain(cuda_fail(e, "crater shape launch"));
                }
            }
            if (bp.any) {
                if (cudaError_t e = launch_boulder_bake(g, t->boulder_width, none, bp.bins, dh,
                                                        bp.status, s, k0, rows, d->waitPolls)) {
                    return drain(cuda_fail(e, "boulder bake launch"));
                }
            }
            if (memory != TG_MEMORY_HOST) {
                continue;
            }
            const size_t y0 = size_t(k0) * kBinCells;
            const size_t y1 = std::min<size_t>(size_t(k0 + rows) * kBinCells, g.height);
            cudaError_t e = cudaEventRecord(d->strips[q], s);
            if (e == cudaSuccess) {
                e = cudaStreamWaitEvent(d->copyStream, d->strips[q], 0);
            }
            if (e == cudaSuccess) {
                e = cudaMemcpyAsync(heights + y0 * g.width, dh + y0 * g.width,
                                    (y1 - y0) * g.width * sizeof(float), cudaMemcpyDeviceToHost,
                                    d->copyStream);
            }
            if (e != cudaSuccess) {
                return drain(cuda_fail(e, "strip copy to host"));
            }
        }
        if (int st = crater_finish(d, cp, s)) {
            return drain(st);
        }
        if (int st = boulder_finish(d, bp, s)) {
            return drain(st);
        }
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        TG_CUDA(cudaStreamSynchronize(d->copyStream), "synchronize");
        bool again = false;
        if (int st = layers_settle(d, &cp, &bp, again)) {
            return st;
        }
        if (!again) {
            return TG_OK;
        }
    }
    return fail(TG_ERROR_MEMORY, "the layers' entries did not fit after growing");
}

int tg_ds_refine(tg_device* d, const float* posts, uint32_t pw, uint32_t ph,
                 const tg_grid* post_grid, const tg_ds_options* o, const tg_grid* grid,
                 float* heights, int memory, void* stream) {
    return tg_ds_refine_window(d, posts, 0, 0, pw, ph, post_grid, o, grid, heights, memory,
                               stream);
}

int tg_ds_refine_window(tg_device* d, const float* posts, int64_t col0, int64_t row0,
                        uint32_t pw, uint32_t ph, const tg_grid* post_grid,
                        const tg_ds_options* o, const tg_grid* grid, float* heights, int memory,
                        void* stream) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (o == nullptr || post_grid == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "options and the post grid are required");
    }
    Grid g, pg;
    if (int s = to_grid(grid, g)) {
        return s;
    }
    if (int s = to_grid(post_grid, pg)) {
        return s;
    }
    if (int s = check_memory(memory)) {
        return s;
    }
    if (!(o->fractal_dimension >= 2.0 && o->fractal_dimension <= 3.0) || !(o->scale >= 0.0) ||
        !std::isfinite(o->scale) || !(o->min_pixel_size >= 0.0)) {
        return fail(TG_ERROR_ARGUMENT, "fractal dimension in [2, 3], scale and min pixel size >= 0");
    }
    if (o->interp > 1u) {
        return fail(TG_ERROR_ARGUMENT, "interp is 0 (bilinear) or 1 (Catmull-Rom)");
    }
    const size_t cells = size_t(g.width) * g.height;
    if (cells == 0) {
        return TG_OK;
    }
    if (pw == 0 || ph == 0 || posts == nullptr || heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "posts and heights are required");
    }
    const bool spline = o->interp == 1u;
    DsTile t{};
    if (!ds_setup(t, pg, o->fractal_dimension, o->scale, o->seed, o->min_pixel_size, spline, g)) {
        return fail(TG_ERROR_ARGUMENT, "the output cells are too coarse for the posts' nodes");
    }
    const cudaStream_t s = stream_of(d, memory, stream);
    const void* dposts = nullptr;
    if (int st = stage_in(d, memory, kDsPosts, posts, size_t(pw) * ph * sizeof(float), &dposts)) {
        return st;
    }
    t.posts = static_cast<const float*>(dposts);
    t.col0 = col0;
    t.row0 = row0;
    t.pw = pw;
    t.ph = ph;
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        TG_CUDA(d->slots[kHeights].reserve(cells * sizeof(float)), "device allocation");
        dh = slot_ptr<float>(d, kHeights);
    }
    t.heights = dh;
    t.pitch = g.width;
    TG_CUDA(d->slots[kStatus].reserve(4 * sizeof(uint32_t)), "allocation");
    t.status = slot_ptr<uint32_t>(d, kStatus);
    TG_CUDA(cudaMemsetAsync(t.status, 0, sizeof(uint32_t), s), "memset");
    TG_CUDA(launch_ds_tiles(t, spline, s), "diamond-square launch");
    TG_CUDA(cudaMemcpyAsync(d->pinnedStatus, t.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
            "copy to host");
    if (int st = copy_heights_back(d, memory, heights, dh, cells)) {
        return st;
    }
    TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    if (d->pinnedStatus[0] & 1u) {
        return fail(TG_ERROR_MEMORY, "a diamond-square block outgrew its shared memory");
    }
    return TG_OK;
}

int tg_philox_probe(tg_device* d, const uint32_t* in, uint32_t n, uint32_t* out,
                    double* normals) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (n == 0) {
        return TG_OK;
    }
    if (in == nullptr || out == nullptr || normals == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "probe buffers are required");
    }
    const void* din = nullptr;
    if (int st = stage_in(d, TG_MEMORY_HOST, kProbeIn, in, size_t(n) * 6 * sizeof(uint32_t),
                          &din)) {
        return st;
    }
    TG_CUDA(d->slots[kProbeHashes].reserve(size_t(n) * 4 * sizeof(uint32_t)), "allocation");
    TG_CUDA(d->slots[kProbeValues].reserve(size_t(n) * sizeof(double)), "allocation");
    TG_CUDA(launch_philox_probe(static_cast<const uint32_t*>(din), n,
                                slot_ptr<uint32_t>(d, kProbeHashes),
                                slot_ptr<double>(d, kProbeValues), d->stream),
            "philox probe");
    TG_CUDA(cudaMemcpyAsync(out, slot_ptr<uint32_t>(d, kProbeHashes), size_t(n) * 16,
                            cudaMemcpyDeviceToHost, d->stream),
            "copy to host");
    TG_CUDA(cudaMemcpyAsync(normals, slot_ptr<double>(d, kProbeValues), size_t(n) * 8,
                            cudaMemcpyDeviceToHost, d->stream),
            "copy to host");
    TG_CUDA(cudaStreamSynchronize(d->stream), "synchronize");
    return TG_OK;
}

int tg_device_counters(tg_device* d, uint64_t* counters, size_t n) {
    if (d == nullptr || (n > 0 && counters == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "device and counters are required");
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    const uint64_t values[2] = {d->craterPairs, d->boulderPairs};
    for (size_t i = 0; i < n && i < 2; ++i) {
        counters[i] = values[i];
    }
    return TG_OK;
}

int tg_measure_alu(tg_device* d, double* lane_ops_per_second) {
    if (int s = check_device(d)) {
        return s;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (lane_ops_per_second == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "output is null");
    }
    TG_CUDA(d->slots[kStatus].reserve(4096 * sizeof(uint32_t)), "allocation");
    double best = 0.0;
    cudaEvent_t start, stop;
    TG_CUDA(cudaEventCreate(&start), "event");
    TG_CUDA(cudaEventCreate(&stop), "event");
    for (int rep = 0; rep < 5; ++rep) {
        uint64_t ops = 0;
        TG_CUDA(cudaEventRecord(start, d->stream), "event");
        TG_CUDA(launch_alu_probe(slot_ptr<uint32_t>(d, kStatus), &ops, d->stream), "alu launch");
        TG_CUDA(cudaEventRecord(stop, d->stream), "event");
        TG_CUDA(cudaEventSynchronize(stop), "event");
        float ms = 0.0f;
        TG_CUDA(cudaEventElapsedTime(&ms, start, stop), "event");
        if (rep > 0 && ms > 0.0f) {
            best = std::max(best, double(ops) / (double(ms) * 1e-3));
        }
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    *lane_ops_per_second = best;
    return TG_OK;
}

}  // extern "C"
