// The relief of older craters under each crater's datum footprint (KernelDatumRelief,
// include/terraingen/layers/kernels/craters.h:1214-1316, run by the reference's
// src/layers/kernels/crater_datums.slang for FitDatumsWithKernel, src/layers/craters/shaping/
// datum_fit.cpp:303-328), on the device.
//
// The lattice is one row per fitted crater and one column per point of its side x side fit
// lattice. A thread takes one point: its offset across the crater's fit footprint, then every
// older crater (index below the fitted one) listed in the cells of each size band within one
// cell of the point, adding the relief each adds there without a datum (CraterRelief). The index
// (band sizes and first cells, cells, entries) is the reference's own, built on the host.
//
// Built with -fmad=false: the offsets and sums round as the reference's -ffp-contract=off build.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "crater_math.cuh"
#include "kernels.h"

using namespace tgb;
using namespace tgb::api;

namespace {

constexpr float kDatumCellSlack = 4.8e-7f;  // craters.h:1241

struct DatumIndex {
    const CraterRecord* records;
    uint32_t nRecords;
    const float* data;
    const float* bandFloats;  // 3 per band: cell size, first column, first row
    const uint32_t* bandCells;  // 3 per band: columns, rows, first cell
    uint32_t nBands;
    const uint32_t* cells;  // 2 per cell: first entry, entries
    uint32_t nCells;
    const uint32_t* entries;
    uint32_t nEntries;
    const uint32_t* targets;
    uint32_t nTargets;
};

// CraterRelief (craters.h:1219): the relief crater `c` adds at (dx, dy) without its datum.
__device__ float crater_relief(const CraterShapeKernel& k, const float* data,
                               const CraterRecord& c, float bound, float dx, float dy) {
    const float squared = dx * dx + dy * dy;
    if (!(squared < bound * bound)) {
        return 0.0f;
    }
    const float distance = crater::shifted_distance(data, c, dx, dy);
    if (!(distance < k.profileReachRadii * 0.5f * c.diameter)) {
        return 0.0f;
    }
    const crater::State s{c.freshDepth, c.freshRim, c.currentDepth, c.currentRim};
    return c.resolution *
           (crater::upslope_height(c, crater::profile_height(k, data, distance, c.diameter, c, s),
                                   dx, dy) +
            crater::peak_relief(k, data, c, s, distance, dx, dy));
}

// KernelCellsNear (craters.h:1251): the first or last cell index within one cell plus slack.
__device__ __forceinline__ int32_t cell_near(float p, float size, float slack, float start,
                                             int32_t count, bool last) {
    return last ? min(int32_t(floorf((p + size + slack) / size) - start), count - 1)
                : max(int32_t(floorf((p - size - slack) / size) - start), 0);
}

__global__ void datum_relief_kernel(const CraterDatumKernel kernel, const DatumIndex ix,
                                    uint32_t width, uint32_t rows, uint32_t firstRow,
                                    float* __restrict__ heights, uint32_t* __restrict__ flags) {
    const uint32_t point = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
    if (point >= width || row >= rows) {
        return;
    }
    const uint32_t target = firstRow + row;
    if (target >= ix.nTargets || ix.targets[target] >= ix.nRecords) {
        atomicOr(flags, 1u);
        return;
    }
    const uint32_t k = ix.targets[target];
    const CraterRecord& fitted = ix.records[k];
    const uint32_t side = kernel.latticeSide;
    const float fitRadius = kernel.fitRadii * 0.5f * fitted.diameter;
    // KernelDatumOffset (craters.h:1236).
    const float dx = fitRadius * ((2.0f * float(point % side) + 1.0f) / float(side) - 1.0f);
    const float dy = fitRadius * ((2.0f * float(point / side) + 1.0f) / float(side) - 1.0f);
    float relief = 0.0f;
    if (dx * dx + dy * dy < fitRadius * fitRadius) {
        const float atX = fitted.x, atXLow = fitted.xLow + dx;
        const float atY = fitted.y, atYLow = fitted.yLow + dy;
        const float px = atX + atXLow;
        const float py = atY + atYLow;
        const float slackX = kDatumCellSlack * fabsf(px);
        const float slackY = kDatumCellSlack * fabsf(py);
        for (uint32_t b = 0; b < ix.nBands; ++b) {
            const float size = ix.bandFloats[3u * b];
            const int32_t across = int32_t(ix.bandCells[3u * b]);
            const int32_t down = int32_t(ix.bandCells[3u * b + 1u]);
            const uint32_t base = ix.bandCells[3u * b + 2u];
            const int32_t c0 = cell_near(px, size, slackX, ix.bandFloats[3u * b + 1u], across, false);
            const int32_t c1 = cell_near(px, size, slackX, ix.bandFloats[3u * b + 1u], across, true);
            const int32_t r0 = cell_near(py, size, slackY, ix.bandFloats[3u * b + 2u], down, false);
            const int32_t r1 = cell_near(py, size, slackY, ix.bandFloats[3u * b + 2u], down, true);
            for (int32_t j = r0; j <= r1; ++j) {
                for (int32_t i = c0; i <= c1; ++i) {
                    const uint32_t cell = base + uint32_t(j * across + i);
                    if (cell >= ix.nCells) {
                        atomicOr(flags, 1u);
                        continue;
                    }
                    const uint32_t first = ix.cells[2u * cell];
                    const uint32_t end = first + ix.cells[2u * cell + 1u];
                    for (uint32_t e = first; e < end && e < ix.nEntries; ++e) {
                        const uint32_t n = ix.entries[e];
                        if (n >= k) {
                            break;
                        }
                        const CraterRecord& r = ix.records[n];
                        const float ox = crater::split_difference(atX, atXLow, r.x, r.xLow);
                        const float oy = crater::split_difference(atY, atYLow, r.y, r.yLow);
                        relief += crater_relief(kernel.shape, ix.data, r, size, ox, oy);
                    }
                }
            }
        }
    }
    float* h = heights + size_t(row) * width + point;
    *h = *h + relief;
}

}  // namespace

extern "C" int tg_crater_datums(tg_device* d, const void* kernel, size_t kernel_bytes,
                                const void* records, uint32_t n_records, const float* data,
                                uint32_t n_data, const float* band_floats, uint32_t n_band_floats,
                                const uint32_t* band_cells, uint32_t n_band_cells,
                                const uint32_t* cells, uint32_t n_cells, const uint32_t* entries,
                                uint32_t n_entries, const uint32_t* targets, uint32_t n_targets,
                                uint32_t width, uint32_t rows, uint32_t first_row, float* heights,
                                int memory, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    if (kernel == nullptr || kernel_bytes != sizeof(CraterDatumKernel)) {
        return fail(TG_ERROR_ARGUMENT, "the datum kernel is %zu bytes", sizeof(CraterDatumKernel));
    }
    CraterDatumKernel k;
    std::memcpy(&k, kernel, sizeof(k));
    if (k.latticeSide == 0u || n_band_floats < 3u * k.bandCount ||
        n_band_cells < 3u * k.bandCount) {
        return fail(TG_ERROR_ARGUMENT, "the datum index does not hold its bands");
    }
    const size_t cellsInLattice = size_t(width) * rows;
    if (cellsInLattice == 0) {
        return TG_OK;
    }
    if (heights == nullptr || targets == nullptr || (n_records > 0 && records == nullptr)) {
        return fail(TG_ERROR_ARGUMENT, "heights, targets and records are required");
    }
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    // Device copies of host arguments, one allocation each, freed on return.
    Buffer bufs[9];
    auto release = [&] {
        for (Buffer& b : bufs) {
            b.release();
        }
    };
    auto stage = [&](int slot, const void* p, size_t bytes) -> const void* {
        if (memory == TG_MEMORY_DEVICE || bytes == 0) {
            return p;
        }
        if (bufs[slot].reserve(bytes) != cudaSuccess ||
            cudaMemcpyAsync(bufs[slot].ptr, p, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            return nullptr;
        }
        return bufs[slot].ptr;
    };
    DatumIndex ix{};
    ix.records = static_cast<const CraterRecord*>(stage(0, records, size_t(n_records) * 144));
    ix.nRecords = n_records;
    ix.data = static_cast<const float*>(stage(1, data, size_t(n_data) * 4));
    ix.bandFloats = static_cast<const float*>(stage(2, band_floats, size_t(n_band_floats) * 4));
    ix.bandCells = static_cast<const uint32_t*>(stage(3, band_cells, size_t(n_band_cells) * 4));
    ix.nBands = k.bandCount;
    ix.cells = static_cast<const uint32_t*>(stage(4, cells, size_t(n_cells) * 4));
    ix.nCells = n_cells / 2u;
    ix.entries = static_cast<const uint32_t*>(stage(5, entries, size_t(n_entries) * 4));
    ix.nEntries = n_entries;
    ix.targets = static_cast<const uint32_t*>(stage(6, targets, size_t(n_targets) * 4));
    ix.nTargets = n_targets;
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        dh = static_cast<float*>(const_cast<void*>(stage(7, heights, cellsInLattice * 4)));
    }
    if ((n_records > 0 && ix.records == nullptr) || dh == nullptr || ix.targets == nullptr) {
        release();
        return fail(TG_ERROR_CUDA, "staging the datum index");
    }
    // A word the kernel sets when the index names a record or cell it does not hold.
    cudaError_t e = bufs[8].reserve(sizeof(uint32_t));
    uint32_t* flags = static_cast<uint32_t*>(bufs[8].ptr);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(flags, 0, sizeof(uint32_t), s);
    }
    if (e == cudaSuccess) {
        const dim3 block(16, 16);
        const dim3 grid((width + 15) / 16, (rows + 15) / 16);
        datum_relief_kernel<<<grid, block, 0, s>>>(k, ix, width, rows, first_row, dh, flags);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && memory == TG_MEMORY_HOST) {
        e = cudaMemcpyAsync(heights, dh, cellsInLattice * 4, cudaMemcpyDeviceToHost, s);
    }
    uint32_t bad = 0;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(&bad, flags, sizeof(bad), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(s);
    }
    release();
    if (e != cudaSuccess) {
        return fail(TG_ERROR_CUDA, "datum relief: %s", cudaGetErrorString(e));
    }
    if (bad != 0u) {
        return fail(TG_ERROR_ARGUMENT, "the datum index names records or cells it does not hold");
    }
    return TG_OK;
}

// --- on a body (crater_body_datums.slang, KernelBodyDatumRelief craters.h:1326) -------------

namespace {

struct BodyDatumIndex {
    const CraterRecord* records;
    uint32_t nRecords;
    const CraterFrame* frames;
    const float* data;
    const float* bounds;    // per record: the reach CraterRelief reads it within (m)
    const uint32_t* lists;  // per row: first entry and entry count
    uint32_t nLists;
    const uint32_t* entries;
    uint32_t nEntries;
    const SplitPoint* positions;  // the strip's lattice points
};

// Each lattice point of a strip gets the relief of its row's craters, each read in its frame
// (BodySplitOffset); points holding no data are left as they are.
__global__ void body_datum_relief_kernel(const CraterShapeKernel k, const BodyDatumIndex ix,
                                         uint32_t width, uint32_t rows, uint32_t firstRow,
                                         const NoData nodata, float* __restrict__ heights,
                                         uint32_t* __restrict__ flags) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = blockIdx.y * blockDim.y + threadIdx.y;
    if (c >= width || r >= rows) {
        return;
    }
    const size_t at = size_t(r) * width + c;
    const float h = heights[at];
    if ((nodata.mode == 1u && isnan(h)) || (nodata.mode == 2u && h == nodata.value)) {
        return;
    }
    const uint32_t row = firstRow + r;
    if (2u * row + 1u >= ix.nLists) {
        atomicOr(flags, 1u);
        return;
    }
    const uint32_t first = ix.lists[2u * row], count = ix.lists[2u * row + 1u];
    const SplitPoint p = ix.positions[at];
    float relief = 0.0f;
    for (uint32_t e = first; e < first + count; ++e) {
        if (e >= ix.nEntries || ix.entries[e] >= ix.nRecords) {
            atomicOr(flags, 1u);
            return;
        }
        const uint32_t n = ix.entries[e];
        const CraterFrame& f = ix.frames[n];
        const crater::Offset o =
            crater::frame_offset(f, crater::split_difference(p.x, p.xLow, f.x, f.xLow),
                                 crater::split_difference(p.y, p.yLow, f.y, f.yLow),
                                 crater::split_difference(p.z, p.zLow, f.z, f.zLow));
        relief += crater_relief(k, ix.data, ix.records[n], ix.bounds[n], o.dx, o.dy);
    }
    heights[at] = h + relief;
}

}  // namespace

extern "C" int tg_crater_body_datums(tg_device* d, const void* kernel, size_t kernel_bytes,
                                     const void* records, uint32_t n_records, const float* data,
                                     uint32_t n_data, const void* frames, const float* bounds,
                                     const uint32_t* lists, uint32_t n_lists,
                                     const uint32_t* entries, uint32_t n_entries,
                                     const void* positions, uint32_t width, uint32_t rows,
                                     uint32_t first_row, float* heights, tg_nodata nodata,
                                     int memory, void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    if (kernel == nullptr || kernel_bytes != sizeof(CraterShapeKernel)) {
        return fail(TG_ERROR_ARGUMENT, "the body datum kernel is %zu bytes",
                    sizeof(CraterShapeKernel));
    }
    if (nodata.mode > 2u) {
        return fail(TG_ERROR_ARGUMENT, "nodata mode must be 0, 1 or 2");
    }
    const size_t points = size_t(width) * rows;
    if (points == 0) {
        return TG_OK;
    }
    if (heights == nullptr || positions == nullptr || lists == nullptr ||
        (n_records > 0 && (records == nullptr || frames == nullptr || bounds == nullptr))) {
        return fail(TG_ERROR_ARGUMENT, "heights, positions, lists and the records are required");
    }
    CraterShapeKernel k;
    std::memcpy(&k, kernel, sizeof(k));
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    Buffer bufs[9];
    auto release = [&] {
        for (Buffer& b : bufs) {
            b.release();
        }
    };
    auto stage = [&](int slot, const void* p, size_t bytes) -> const void* {
        if (memory == TG_MEMORY_DEVICE || bytes == 0) {
            return p;
        }
        if (bufs[slot].reserve(bytes) != cudaSuccess ||
            cudaMemcpyAsync(bufs[slot].ptr, p, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            return nullptr;
        }
        return bufs[slot].ptr;
    };
    BodyDatumIndex ix{};
    ix.records = static_cast<const CraterRecord*>(stage(0, records, size_t(n_records) * 144));
    ix.nRecords = n_records;
    ix.frames = static_cast<const CraterFrame*>(stage(1, frames, size_t(n_records) * 52));
    ix.data = static_cast<const float*>(stage(2, data, size_t(n_data) * 4));
    ix.bounds = static_cast<const float*>(stage(3, bounds, size_t(n_records) * 4));
    ix.lists = static_cast<const uint32_t*>(stage(4, lists, size_t(n_lists) * 4));
    ix.nLists = n_lists;
    ix.entries = static_cast<const uint32_t*>(stage(5, entries, size_t(n_entries) * 4));
    ix.nEntries = n_entries;
    ix.positions = static_cast<const SplitPoint*>(stage(6, positions, points * 24));
    float* dh = heights;
    if (memory == TG_MEMORY_HOST) {
        dh = static_cast<float*>(const_cast<void*>(stage(7, heights, points * 4)));
    }
    if ((n_records > 0 && (ix.records == nullptr || ix.frames == nullptr)) || dh == nullptr ||
        ix.lists == nullptr || ix.positions == nullptr) {
        release();
        return fail(TG_ERROR_CUDA, "staging the body datum index");
    }
    cudaError_t e = bufs[8].reserve(sizeof(uint32_t));
    uint32_t* flags = static_cast<uint32_t*>(bufs[8].ptr);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(flags, 0, sizeof(uint32_t), s);
    }
    if (e == cudaSuccess) {
        const dim3 block(16, 16);
        const dim3 grid((width + 15) / 16, (rows + 15) / 16);
        body_datum_relief_kernel<<<grid, block, 0, s>>>(k, ix, width, rows, first_row,
                                                         NoData{nodata.mode, nodata.value}, dh,
                                                         flags);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && memory == TG_MEMORY_HOST) {
        e = cudaMemcpyAsync(heights, dh, points * 4, cudaMemcpyDeviceToHost, s);
    }
    uint32_t bad = 0;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(&bad, flags, sizeof(bad), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(s);
    }
    release();
    if (e != cudaSuccess) {
        return cuda_fail(e, "body datum relief");
    }
    if (bad != 0u) {
        return fail(TG_ERROR_ARGUMENT, "the body datum lists name a row, entry or record out of range");
    }
    return TG_OK;
}
