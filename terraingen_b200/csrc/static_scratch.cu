// Boulder baking without allocation: the same pipeline as tg_boulders_bake (count, scan,
// scatter, bake; boulders.cu), its scratch memory held in one file-scope device array instead of
// memory the library allocates.
//
// Some callers cannot allocate GPU memory while they evaluate terrain: a streaming renderer's
// frame thread, where cudaMalloc or cudaFree would synchronize the whole device and stall the
// frame, and hosts that fix their GPU memory at start-up and allow no growth afterwards. This
// entry point serves them: it takes the caller's device buffers and a stream and allocates
// nothing, at the price of a fixed capacity and a shared scratch array.
//
// The array is part of the library image: every GPU that loads the library holds it, all
// kStaticScratchBytes of it, until the process exits. Calls share it, and it keeps what the last
// call left, so every call clears the parts that must start at zero; two calls whose work
// overlaps on the GPU (different streams, or different host threads) race on it and must not
// overlap.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/tgb200.h"
#include "kernels.h"

namespace tgb {
namespace {

// 16 MiB: the bins of a grid up to kStaticMaxCells cells, the windows of up to
// kStaticMaxBoulders boulders and up to kStaticMaxEntries binned boulders.
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr uint32_t kStaticMaxBoulders = 1u << 16;
constexpr uint32_t kStaticMaxBins = 1u << 15;
constexpr uint32_t kStaticMaxEntries = 196608;

static __device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

// Byte offsets of the scratch's parts, each 256-byte aligned.
constexpr size_t align256(size_t b) {
    return (b + 255) & ~size_t(255);
}
constexpr size_t kOffStatus = 0;
constexpr size_t kOffCounts = 256;
constexpr size_t kOffCursor = kOffCounts + align256((kStaticMaxBins + 1) * sizeof(uint32_t));
constexpr size_t kOffScan = kOffCursor + align256(kStaticMaxBins * sizeof(uint32_t));
constexpr size_t kScanWords = 64;  // scan_scratch_words(kStaticMaxBins) fits
constexpr size_t kOffWindows = kOffScan + align256(kScanWords * sizeof(uint32_t));
constexpr size_t kOffEntries = kOffWindows + align256(kStaticMaxBoulders * sizeof(int4));
constexpr size_t kEnd = kOffEntries + size_t(kStaticMaxEntries) * sizeof(BoulderEntry);
static_assert(kEnd <= kStaticScratchBytes, "the static scratch parts must fit the array");

// The array's device address on each device, found once per device with that device current.
// In host code `g_scratch` names a host-side stand-in, not device memory, so kernels must be given
// this address instead.
std::mutex g_setup;
void* g_address[64] = {};

const char* scratch_address(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup);
    if (device < 0 || device >= 64) {
        return "device ordinal out of range";
    }
    if (g_address[device] == nullptr) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || ptr == nullptr) {
            cudaGetLastError();
            return "cudaGetSymbolAddress of the static scratch failed";
        }
        g_address[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_address[device]);
    return nullptr;
}

}  // namespace
}  // namespace tgb

using namespace tgb;

extern "C" int tg_boulders_bake_static(const void* boulders, uint32_t n, double width,
                                       const tg_grid* grid, float* heights, tg_nodata nodata,
                                       void* stream, char* error, size_t error_capacity) {
    auto fail = [&](int status, const char* message) {
        if (error != nullptr && error_capacity > 0) {
            size_t i = 0;
            for (; message[i] != '\0' && i + 1 < error_capacity; ++i) {
                error[i] = message[i];
            }
            error[i] = '\0';
        }
        return status;
    };
    if (grid == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "grid is null");
    }
    if (grid->row_rotation != 0.0 || grid->col_rotation != 0.0) {
        return fail(TG_ERROR_UNSUPPORTED, "rotated grids are not supported");
    }
    if (!(grid->pixel_width != 0.0) || !(grid->pixel_height != 0.0)) {
        return fail(TG_ERROR_ARGUMENT, "grid transform must be invertible");
    }
    if (nodata.mode > 2u || !(width >= 0.0)) {
        return fail(TG_ERROR_ARGUMENT, "nodata mode or width out of range");
    }
    const size_t cells = size_t(grid->width) * grid->height;
    if (cells == 0 || n == 0) {
        return fail(TG_OK, "");
    }
    if (boulders == nullptr || heights == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "boulders and heights are required");
    }
    if (reinterpret_cast<uintptr_t>(boulders) % 8u != 0u ||
        reinterpret_cast<uintptr_t>(heights) % 4u != 0u) {
        return fail(TG_ERROR_ARGUMENT, "boulders must be 8-byte and heights 4-byte aligned");
    }
    const Grid g{grid->width,        grid->height,   grid->origin_x,    grid->pixel_width,
                 grid->row_rotation, grid->origin_y, grid->col_rotation, grid->pixel_height};
    BoulderBins bins{};
    bins.binsX = (g.width + kBinCells - 1) / kBinCells;
    bins.binsY = (g.height + kBinCells - 1) / kBinCells;
    const uint32_t nbins = bins.binsX * bins.binsY;
    if (n > kStaticMaxBoulders || nbins > kStaticMaxBins ||
        scan_scratch_words(nbins) > kScanWords) {
        return fail(TG_ERROR_ARGUMENT,
                    "beyond the static scratch: at most 65536 boulders and 32768 bins of 32x32 "
                    "cells");
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return fail(TG_ERROR_CUDA, "cudaGetDevice failed");
    }
    unsigned char* base = nullptr;
    if (const char* why = scratch_address(device, &base)) {
        return fail(TG_ERROR_CUDA, why);
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* status = reinterpret_cast<uint32_t*>(base + kOffStatus);
    bins.counts = reinterpret_cast<uint32_t*>(base + kOffCounts);
    bins.cursor = reinterpret_cast<uint32_t*>(base + kOffCursor);
    bins.windows = reinterpret_cast<int4*>(base + kOffWindows);
    bins.entries = reinterpret_cast<BoulderEntry*>(base + kOffEntries);
    bins.capacity = kStaticMaxEntries;
    uint32_t* scan = reinterpret_cast<uint32_t*>(base + kOffScan);
    const BoulderRecord* rec = static_cast<const BoulderRecord*>(boulders);
    // What the last call left: counts, cursors and the status start at zero.
    if (cudaMemsetAsync(status, 0, 256, s) != cudaSuccess ||
        cudaMemsetAsync(bins.counts, 0, (size_t(nbins) + 1) * sizeof(uint32_t), s) !=
            cudaSuccess ||
        cudaMemsetAsync(bins.cursor, 0, size_t(nbins) * sizeof(uint32_t), s) != cudaSuccess ||
        launch_boulder_count(rec, n, g, width, bins, s) != cudaSuccess ||
        launch_exclusive_scan(bins.counts, nbins, scan, s) != cudaSuccess) {
        cudaGetLastError();
        return fail(TG_ERROR_CUDA, "a launch of the static bake failed");
    }
    // Beyond the scratch's capacity (the scan's total, checked on the device) the scatter and the
    // bake write nothing and the bake sets flag 4, so the heights are left as they were.
    const NoData nd{nodata.mode, nodata.value};
    if (launch_boulder_scatter(rec, n, bins, s) != cudaSuccess ||
        launch_boulder_bake(g, width, nd, bins, heights, status, s) != cudaSuccess) {
        cudaGetLastError();
        return fail(TG_ERROR_CUDA, "a launch of the static bake failed");
    }
    uint32_t flags = 0;
    if (cudaMemcpyAsync(&flags, status, sizeof(flags), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return fail(TG_ERROR_CUDA, "reading the static bake's status failed");
    }
    if (flags & 4u) {
        return fail(TG_ERROR_MEMORY,
                    "the boulders cover more bin entries than the static scratch holds (196608); "
                    "the heights are unchanged");
    }
    if (flags & 2u) {
        return fail(TG_ERROR_TIMEOUT, "a boulder bin's staged copy did not arrive");
    }
    return fail(TG_OK, "");
}
