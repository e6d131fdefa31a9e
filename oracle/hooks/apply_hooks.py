"""Builds the reference sources with libtgb200's hooks at its CPU-only stages, for the drop-in
build (oracle/_ref/libtgref_cuda.so): test infrastructure, never part of the product.

The hooks are the lines a TerrainGen maintainer adds at those stages: synthetic sources on a
grid through tg_noise_source, boulder domes through tg_boulders_bake, diamond-square on a grid
through tg_ds_refine, each when the evaluation runs on Backend::Cuda
(tgb200_hooks_active, set by the harness for backend 1) and the stage's options are the ones the
library restates; otherwise the reference's own code runs as it is. The reference's files are
read from the checkout, each hook block (this file's own code) is inserted at the first line of
the function it hooks, and the result is written to oracle/_ref/hooked/src/<same path>; nothing of
the reference is copied into the repository.

    python oracle/hooks/apply_hooks.py <reference checkout> <output directory>
"""

from __future__ import annotations

import sys
from pathlib import Path

INCLUDE = '#include "tgb200_hooks.h"\n'

# (file, the function's opening line, the hook block placed right after it)
HOOKS = [
    ("sources/synthetic_source.cpp",
     "void SyntheticSource::FillSamples(SampleBlock& samples, double spacing, unsigned threads) const {",
     """
    // libtgb200: a grid of a plane source on the device (bit-exact with the CPU fill).
    if (Raster<float>* grid = samples.Grid(); grid != nullptr && !m_posts &&
                                              !m_surface.IsBody() && tgb200_hooks_active() &&
                                              !m_fractals.empty()) {
        const tg_grid g = tgb200_grid(*grid);
        if (tg_noise_source(tgb200_device(), m_fractals.data(),
                            static_cast<uint32_t>(m_fractals.size()), m_elevation, &g,
                            grid->Values().data(), TG_MEMORY_HOST, nullptr) == TG_OK) {
            return;
        }
    }
"""),
    ("layers/boulders/boulder_relief.cpp",
     "void BoulderLayer::ApplySamples(SampleBlock& samples, const LayerContext& context) const {",
     """
    // libtgb200: domes without fillets, facets or shapes on a plane grid, baked on the device.
    if (Raster<float>* grid = samples.Grid();
        grid != nullptr && context.backend == Backend::Cuda && tgb200_hooks_active() &&
        !m_surface.IsBody() && m_options.rendering.relief == BoulderRelief::Dome &&
        m_options.fillet.heightShare <= 0.0 && m_options.ventifacts.share <= 0.0) {
        const double at = samples.ResolvedSpacing(context.spacing, m_surface);
        const std::vector<Boulder> found =
            ReliefBoulders(samples.Bounds(), at, context.ground, context.threads);
        const std::vector<Relief> reliefs = PrepareRelief(found, at, true);
        std::vector<tg_boulder> domes;
        bool plain = true;
        for (const Relief& r : reliefs) {
            plain = plain && r.Shape() == nullptr && r.contacts.empty();
            if (r.rock) {
                domes.push_back({r.boulder->x, r.boulder->y, r.boulder->diameter,
                                 r.boulder->ExposedHeight(), r.weight});
            }
        }
        const tg_grid g = tgb200_grid(*grid);
        if (plain && tg_boulders_bake(tgb200_device(), domes.data(),
                                      static_cast<uint32_t>(domes.size()), at, &g,
                                      grid->Values().data(), tgb200_nodata(*grid),
                                      TG_MEMORY_HOST, nullptr) == TG_OK) {
            return;
        }
    }
"""),
    ("sources/diamond_square.cpp",
     "void DiamondSquareUpsampler::FillSamples(const PostLattice& posts, SampleBlock& samples,",
     None),  # the opening spans two lines; the block goes after the brace (see below)
]

DS_OPEN_TAIL = "                                         double spacing, unsigned threads) const {"
DS_BLOCK = """
    // libtgb200: refinement of a grid at the grid's own spacing, with F and the scale given, on
    // the device; the posts it reads come from the lattice with a margin.
    if (Raster<float>* grid = samples.Grid();
        grid != nullptr && tgb200_hooks_active() && m_options.fractalDimension &&
        m_options.scale && tgb200_at_grid_spacing(*grid, spacing)) {
        std::vector<float> window;
        int64_t col0 = 0, row0 = 0;
        tg_grid lattice{};
        const tg_grid out = tgb200_grid(*grid);
        if (tgb200_post_window(posts, *grid, 16, window, col0, row0, lattice)) {
            const uint32_t interp =
                m_options.interp == DiamondSquareInterp::CatmullRom ? 1u : 0u;
            const tg_ds_options o{*m_options.fractalDimension, *m_options.scale, interp,
                                  m_options.seed, m_options.minPixelSize};
            if (tg_ds_refine_window(tgb200_device(), window.data(), col0, row0, lattice.width,
                                    lattice.height, &lattice, &o, &out, grid->Values().data(),
                                    TG_MEMORY_HOST, nullptr) == TG_OK) {
                return;
            }
        }
    }
"""


def main(ref: Path, out: Path) -> None:
    for path, opening, block in HOOKS:
        text = (ref / "src" / path).read_text()
        if block is None:
            anchor = opening + "\n" + DS_OPEN_TAIL
            block = DS_BLOCK
        else:
            anchor = opening
        if text.count(anchor) != 1:
            raise SystemExit(f"{path}: hook anchor not found once")
        text = text.replace(anchor, anchor + block, 1)
        # The include goes after the file's first include line.
        first = text.index("#include")
        end = text.index("\n", first) + 1
        text = text[:end] + INCLUDE + text[end:]
        dest = out / "src" / path
        dest.parent.mkdir(parents=True, exist_ok=True)
        dest.write_text(text)


if __name__ == "__main__":
    main(Path(sys.argv[1]), Path(sys.argv[2]))
