// oracle/hooks/tgb200_hooks.cpp - test infrastructure only: the glue of tgb200_hooks.h, linked
// into the drop-in build of the reference (oracle/_ref/libtgref_cuda.so).
#include "tgb200_hooks.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>

namespace {
std::atomic<bool> g_active{false};
std::atomic<long> g_calls{0};
std::mutex g_open;
tg_device* g_device = nullptr;
}  // namespace

bool tgb200_hooks_active() {
    return g_active.load();
}

void tgb200_set_hooks_active(bool active) {
    g_active.store(active);
}

long tgb200_hook_calls() {
    return g_calls.load();
}

tg_device* tgb200_device() {
    ++g_calls;
    std::lock_guard<std::mutex> lock(g_open);
    if (g_device == nullptr && tg_open(0, &g_device) != TG_OK) {
        throw std::runtime_error(std::string("tgb200: ") + tg_last_error());
    }
    return g_device;
}

tg_grid tgb200_grid(const terraingen::Raster<float>& raster) {
    const terraingen::GeoTransform& t = raster.Transform();
    return tg_grid{static_cast<uint32_t>(raster.Width()), static_cast<uint32_t>(raster.Height()),
                   t.originX, t.pixelWidth, t.rowRotation, t.originY, t.colRotation,
                   t.pixelHeight};
}

tg_nodata tgb200_nodata(const terraingen::Raster<float>& raster) {
    const auto& value = raster.NoData();
    if (!value) {
        return tg_nodata{0u, 0.0f};
    }
    if (std::isnan(*value)) {
        return tg_nodata{1u, 0.0f};
    }
    return tg_nodata{2u, *value};
}

bool tgb200_at_grid_spacing(const terraingen::Raster<float>& raster, double spacing) {
    const terraingen::GeoTransform& t = raster.Transform();
    const double cell = std::fmax(std::fabs(t.pixelWidth), std::fabs(t.pixelHeight));
    return std::fabs(spacing - cell) <= 1e-9 * cell;
}

bool tgb200_post_window(const terraingen::PostLattice& lattice,
                        const terraingen::Raster<float>& raster, int margin,
                        std::vector<float>& posts, int64_t& first_col, int64_t& first_row,
                        tg_grid& grid) {
    const terraingen::GeoTransform p = lattice.Transform();
    const terraingen::GeoTransform& r = raster.Transform();
    if (p.rowRotation != 0.0 || p.colRotation != 0.0 || r.rowRotation != 0.0 ||
        r.colRotation != 0.0) {
        return false;
    }
    // The raster's bounds in the lattice's post coordinates (post k at the center of cell k).
    const double xa = r.originX, xb = r.originX + double(raster.Width()) * r.pixelWidth;
    const double ya = r.originY, yb = r.originY + double(raster.Height()) * r.pixelHeight;
    const double c0 = (std::fmin(xa, xb) - p.originX) / p.pixelWidth;
    const double c1 = (std::fmax(xa, xb) - p.originX) / p.pixelWidth;
    const double r0 = (std::fmin(ya, yb) - p.originY) / p.pixelHeight;
    const double r1 = (std::fmax(ya, yb) - p.originY) / p.pixelHeight;
    int64_t col0 = int64_t(std::floor(std::fmin(c0, c1))) - margin;
    int64_t col1 = int64_t(std::ceil(std::fmax(c0, c1))) + margin;
    int64_t row0 = int64_t(std::floor(std::fmin(r0, r1))) - margin;
    int64_t row1 = int64_t(std::ceil(std::fmax(r0, r1))) + margin;
    // A bounded lattice repeats its edge posts beyond its extent, as the device repeats the
    // window's: the window stops at the extent.
    if (const auto extent = lattice.Extent()) {
        col0 = std::max(col0, int64_t(extent->colBegin));
        col1 = std::min(col1, int64_t(extent->colEnd));
        row0 = std::max(row0, int64_t(extent->rowBegin));
        row1 = std::min(row1, int64_t(extent->rowEnd));
        if (col0 >= col1 || row0 >= row1) {
            col0 = std::min(col0, int64_t(extent->colEnd) - 1);
            row0 = std::min(row0, int64_t(extent->rowEnd) - 1);
            col1 = col0 + 1;
            row1 = row0 + 1;
        }
    }
    const size_t width = size_t(col1 - col0), height = size_t(row1 - row0);
    posts.assign(width * height, 0.0f);
    lattice.Read(col0, row0, width, height, terraingen::Span<float>(posts.data(), posts.size()));
    first_col = col0;
    first_row = row0;
    // The whole lattice's transform: its post (0, 0) anchors the refinement's node frame.
    grid = tg_grid{uint32_t(width), uint32_t(height), p.originX, p.pixelWidth, 0.0, p.originY,
                   0.0, p.pixelHeight};
    return true;
}
