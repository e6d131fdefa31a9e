// oracle/hooks/tgb200_hooks.h - test infrastructure only, never part of the product.
//
// The glue the hook blocks of oracle/hooks/apply_hooks.py call from inside the reference's
// sources (the lines a TerrainGen maintainer adds at its CPU-only stages): the device, whether the
// evaluation runs on Backend::Cuda, and conversions of the reference's rasters and post lattices
// to the C ABI's grids.
#pragma once

#include <cstdint>
#include <vector>

#include "tgb200.h"
#include "terraingen/raster/raster.h"
#include "terraingen/sources/upsampling.h"

// Whether the current evaluation asked for Backend::Cuda (the harness sets it around
// Terrain::Evaluate; sources are not told the backend).
bool tgb200_hooks_active();
void tgb200_set_hooks_active(bool active);

// The device the hooks run on, opened on first use; every call counts as one hooked stage.
tg_device* tgb200_device();
long tgb200_hook_calls();

// A raster's grid and no-data marking as the C ABI takes them.
tg_grid tgb200_grid(const terraingen::Raster<float>& raster);
tg_nodata tgb200_nodata(const terraingen::Raster<float>& raster);

// Whether `spacing` is the raster's own cell size (the refinement's levels follow the spacing).
bool tgb200_at_grid_spacing(const terraingen::Raster<float>& raster, double spacing);

// The lattice's posts over the raster's bounds and `margin` posts around (within its extent,
// for a bounded lattice), into `posts` (row 0 north): columns first_col.. and rows first_row.. of
// the lattice, whose transform goes to `grid`; false for a rotated lattice or raster.
bool tgb200_post_window(const terraingen::PostLattice& lattice,
                        const terraingen::Raster<float>& raster, int margin,
                        std::vector<float>& posts, int64_t& first_col, int64_t& first_row,
                        tg_grid& grid);
