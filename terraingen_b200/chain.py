"""Raster patches chained with seams on the device: SourceChain::FillSamples over a grid
(src/sources/source_chain.cpp:154-192) for sources that are rasters on windows of one grid.

The chain [P0, P1, ..., Pn-1] reads P0 where it has data; each later patch Pk fills the cells the
chain before it leaves without data, corrected by the seam field of the link (Pk's prefix, Pk).
As in SourceChain::Seam (source_chain.cpp:144-152), the link's lattice is the grid of the source
just before Pk (the window of P(k-1)) padded by ceil(reach / spacing) + 3 posts (SeamLattice,
source_chain.cpp:94-114), and the prefix is sampled on it as the chain so far has filled the grid.
Every step runs on the device through the C ABI: tg_seam_samples (SampleSources),
tg_seam_solve (BuildSeamField) and tg_seam_fill (FillGridGaps).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

from .device import Device, GridSpec

SEAM_BORDER_POSTS = 3  # source_chain.cpp:26
SEAM_REACH_DECAYS = 3.0  # a Height / Slope seam reaches 3 decay lengths


@dataclass(frozen=True)
class Window:
    """Cells [col0, col0 + width) x [row0, row0 + height) of a grid."""

    col0: int
    row0: int
    width: int
    height: int

    def grid(self, grid: GridSpec) -> GridSpec:
        return GridSpec(self.width, self.height, grid.x0 + self.col0 * grid.pixel,
                        grid.y0 - self.row0 * grid.pixel, grid.pixel)

    def slices(self):
        return (slice(self.row0, self.row0 + self.height),
                slice(self.col0, self.col0 + self.width))


@dataclass(frozen=True)
class Seams:
    """ChainSeams (source_chain.h:38): mode "none", "feather", "height" or "slope"."""

    mode: str = "height"
    width: float = 50.0
    decay_length: float = 50.0
    levels: int = 4
    sweeps: int = 2
    coarsest_sweeps: int = 20

    @property
    def reach(self) -> float:
        if self.mode == "feather":
            return self.width
        if self.mode in ("height", "slope"):
            return SEAM_REACH_DECAYS * self.decay_length
        return 0.0


class PatchChain:
    """Patches on windows of `grid` joined by `seams`, with device buffers sized once.

    compose(patches) takes each patch's heights (a device tensor of its window's shape) and
    returns the grid's heights (a device tensor, NaN where no patch has data). Statistics of
    the last compose's seam solves are in `solves`.
    """

    def __init__(self, device: Device, grid: GridSpec, windows: list[Window], seams: Seams):
        import torch

        self.device, self.grid, self.windows, self.seams = device, grid, windows, seams
        self.pad = math.ceil(seams.reach / grid.pixel) + SEAM_BORDER_POSTS
        shape = (grid.height, grid.width)
        nan = float("nan")
        self.heights = torch.full(shape, nan, dtype=torch.float32, device="cuda")
        # Each later patch on the whole grid (no data off its window), filled in place.
        self.later = [torch.full(shape, nan, dtype=torch.float32, device="cuda")
                      for _ in windows[1:]]
        posts = max((w.width + 2 * self.pad) * (w.height + 2 * self.pad) for w in windows[:-1]) \
            if len(windows) > 1 else 0
        self._data = torch.empty(posts, dtype=torch.uint8, device="cuda")
        self._diff = torch.empty(posts, dtype=torch.float32, device="cuda")
        self._field = torch.empty(posts, dtype=torch.float32, device="cuda")
        self.solves: list[dict] = []

    def lattice(self, k: int) -> tuple[Window, GridSpec]:
        """The lattice of link k (k >= 1): the window of patch k - 1 padded on every side."""
        w = self.windows[k - 1]
        win = Window(w.col0 - self.pad, w.row0 - self.pad, w.width + 2 * self.pad,
                     w.height + 2 * self.pad)
        return win, win.grid(self.grid)

    def compose(self, patches, events=None):
        """The chain's heights on the grid. With `events` (a list), appends per link the CUDA
        events (start, sampled, solved, filled) recorded on the current stream."""
        import torch

        dev, s = self.device, self.seams
        stream = torch.cuda.current_stream()
        self.heights.fill_(float("nan"))
        self.heights[self.windows[0].slices()].copy_(patches[0])
        self.solves = []
        for k in range(1, len(self.windows)):
            later = self.later[k - 1]
            later[self.windows[k].slices()].copy_(patches[k])
            win, lgrid = self.lattice(k)
            n = win.width * win.height
            data = self._data[:n].view(win.height, win.width)
            diff = self._diff[:n].view(win.height, win.width)
            field = self._field[:n].view(win.height, win.width)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if events is not None \
                else None
            if ev:
                ev[0].record(stream)
            dev.seam_samples(self.heights, later, self.grid, win.col0, win.row0, win.width,
                             win.height, data=data, difference=diff)
            if ev:
                ev[1].record(stream)
            _, stats = dev.seam_solve(data, diff, self.grid.pixel, self.grid.pixel, s.mode,
                                      width=s.width, decay_length=s.decay_length, field=field,
                                      levels=s.levels, sweeps=s.sweeps,
                                      coarsest_sweeps=s.coarsest_sweeps)
            if ev:
                ev[2].record(stream)
            wk = self.windows[k]
            dev.seam_fill(field, lgrid, later, self.grid, self.heights,
                          window=(wk.col0, wk.row0, wk.width, wk.height))
            if ev:
                ev[3].record(stream)
                events.append(ev)
            self.solves.append(stats)
        return self.heights
