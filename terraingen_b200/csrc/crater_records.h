// The device record builder's inputs (crater_records.cu): what tg_crater_batch's host side makes
// before the records themselves, the batch's craters in apply order with the per-crater data only
// the host's libm gives (wall terraces, massif peaks), and the constants every record reads.
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "../../include/tgb200.h"

namespace tgb {

// One candidate crater of a batch, in the population's draw order (the device puts them in
// CraterApplyOrder, apply_options.cpp:96).
struct RecordCrater {
    double x, y, diameter;
    double age;             // Gyr (the apply order's first key)
    double erosion;         // the share of the fresh depth and rim left (FreshnessDegradation)
    uint64_t id;
    uint32_t extraOffset;   // its terrace floats, then its peak floats, in the plan's extras
    uint32_t terraceFloats;
    uint32_t extraFloats;
    uint16_t terraceCount;  // AppendKernelTerraces' benches (0: none)
    uint16_t peakCount;     // AppendKernelPeaks' massifs (0: none)
};
static_assert(sizeof(RecordCrater) == 64, "RecordCrater is 64 bytes");

// The constants of a batch's records (MakeCraterKernelBatch under the batch's shaping).
struct RecordConstants {
    double originX, originY, pixelWidth, pixelHeight, rowRotation, colRotation;
    double width, height;       // the grid's cells, as doubles (ClampIndex's bounds)
    double spacing;             // the larger pixel side (the resolution weight's unit)
    double reachRadii;          // the profile's reach in radii
    double freshDepth, freshRim;
    double outlinePower[11];    // k^-1.5 for harmonics k = 2..12 (IrregularOutline's law)
    double outlineScale;        // sqrt(2 / sum of k^-3)
    uint32_t irregular;         // DefaultCraterApply's outlines, terraces and peaks
    uint32_t irregularitySeed, noiseSeed, textureKeySeed;
};

namespace host {

// tg_crater_batch up to its records, less the apply order: the population drawn over the grid's
// bounds, the candidates, and for every candidate that carries them its wall terraces and massif
// peaks (built as tg_crater_batch builds them); `kernel` (when not null) receives the batch's
// CraterShapeKernel. The candidates, in draw order, go where `place(n)` says (room for n, or
// null to refuse: TG_ERROR_MEMORY), their extras into `extras`. `n` receives their number.
// Returns a TG_* status.
int record_plan(const tg_crater_population& spec, const tg_crater_shaping& shaping,
                const tg_grid& grid, void* kernel, RecordConstants& constants,
                const std::function<RecordCrater*(size_t)>& place, size_t& n,
                std::vector<float>& extras);

}  // namespace host
}  // namespace tgb
