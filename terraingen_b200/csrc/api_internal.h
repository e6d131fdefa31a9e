// Internals of the C ABI shared by its units (api.cu, batch_api.cu): error reporting, growable
// device buffers, the device handle and argument checks.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/tgb200.h"
#include "kernels.h"

namespace tgb {
namespace api {

// Records the message for tg_last_error (thread-local) and returns `status`.
int fail(int status, const char* format, ...);
int cuda_fail(cudaError_t err, const char* what);

#define TG_CUDA(call, what)                    \
    do {                                       \
        const cudaError_t e_ = (call);         \
        if (e_ != cudaSuccess) {               \
            return ::tgb::api::cuda_fail(e_, what); \
        }                                      \
    } while (0)

// One growable device allocation.
struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;

    cudaError_t reserve(size_t need) {
        if (need <= bytes) {
            return cudaSuccess;
        }
        if (ptr != nullptr) {
            cudaFree(ptr);
            ptr = nullptr;
            bytes = 0;
        }
        // Grow by half again to amortise repeated growth, except for buffers of a GiB or more,
        // which are sized exactly (a grid of billions of cells).
        const size_t size = need < (size_t(1) << 30) ? need + need / 2 : need;
        const cudaError_t err = cudaMalloc(&ptr, size);
        if (err == cudaSuccess) {
            bytes = size;
        }
        return err;
    }
    void release() {
        if (ptr != nullptr) {
            cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
};

enum Slot {
    kHeights,
    kXs,
    kYs,
    kXLows,
    kYLows,
    kRecords,
    kData,
    kFootprints,
    kHeads,
    kEntries,
    kCounts,
    kCursor,
    kBoxes,
    kCulls,
    kBinEntries,
    kHarmonics,
    kScan,
    kStatus,
    kBoulders,
    kBoulderWindows,
    kBoulderEntries,
    kDsPosts,
    kProbeIn,
    kProbeHashes,
    kProbeValues,
    kFrames,
    kPoints,
    kBoulderCounts,
    kBoulderCursor,
    kBoulderStatus,
    kPairStart,
    kExtrasMark,
    kExtrasList,
    kRecordCraters,  // the device record builder's plan: craters, then extras
    kRecordCounts,   // its records and floats per crater, then their scans
    kRecordSort,     // the apply order's keys, orders and sort scratch
    kSlotCount
};

int check_device(tg_device* d);
int check_memory(int memory);
int to_grid(const tg_grid* g, Grid& out);

}  // namespace api
}  // namespace tgb

struct tg_device {
    int ordinal = 0;
    cudaStream_t stream = nullptr;
    // Host-memory inputs copied on their own stream, to overlap the first kernels of a call.
    cudaStream_t copyStream = nullptr;
    cudaEvent_t copied = nullptr;
    cudaEvent_t strips[8] = {};  // a call's strips of output rows, ready to copy out
    std::mutex mutex;
    std::string name;
    tgb::api::Buffer slots[tgb::api::kSlotCount];
    uint32_t* pinnedStatus = nullptr;  // 16 host-pinned words read back after the layers
    // The device record builder's page-locked staging (tg_crater_batch_device).
    void* recordStage = nullptr;
    size_t recordStageBytes = 0;
    // (cell, crater) and (cell, boulder) pairs evaluated by the last shaping and bake.
    unsigned long long craterPairs = 0, boulderPairs = 0;
    // Polls of a staged copy before the binned kernels give up on it (tg_set_wait_limit).
    uint32_t waitPolls = tgb::kWaitPolls;
    // The seam solve's scratch, kept across calls and released by tg_close.
    void* seams = nullptr;
    void (*releaseSeams)(void*) = nullptr;
};
