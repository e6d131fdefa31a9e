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

    def __init__(self, device: Device, grid: GridSpec, windows: list[Window], seams: Seams,
                 tensors: str = "cuda", links=None):
        import torch

        self.device, self.grid, self.windows, self.seams = device, grid, windows, seams
        self.pad = math.ceil(seams.reach / grid.pixel) + SEAM_BORDER_POSTS
        shape = (grid.height, grid.width)
        nan = float("nan")
        self.heights = torch.full(shape, nan, dtype=torch.float32, device=tensors)
        # Each later patch on the whole grid (no data off its window), filled in place; with
        # `links` only those links' patches are held.
        self._links = list(range(1, len(windows))) if links is None else list(links)
        self.later = {k: torch.full(shape, nan, dtype=torch.float32, device=tensors)
                      for k in self._links}
        posts = max(((self.windows[k - 1].width + 2 * self.pad) *
                     (self.windows[k - 1].height + 2 * self.pad) for k in self._links), default=0)
        self._data = torch.empty(posts, dtype=torch.uint8, device=tensors)
        self._diff = torch.empty(posts, dtype=torch.float32, device=tensors)
        self._field = torch.empty(posts, dtype=torch.float32, device=tensors)
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

        self.heights.fill_(float("nan"))
        self.heights[self.windows[0].slices()].copy_(patches[0])
        self.solves = []
        for k in range(1, len(self.windows)):
            self.link(k, patches[k], events)
        return self.heights

    def link(self, k: int, patch, events=None):
        """Link k (k >= 1) on `self.heights`, which must hold the chain's heights after link
        k - 1 on the lattice of link k and on patch k's window (SourceChain::Seam and
        FillGridGaps for patch k): samples, solve, fill."""
        import torch

        dev, s = self.device, self.seams
        later = self.later[k]
        later[self.windows[k].slices()].copy_(patch)
        win, lgrid = self.lattice(k)
        n = win.width * win.height
        data = self._data[:n].view(win.height, win.width)
        diff = self._diff[:n].view(win.height, win.width)
        field = self._field[:n].view(win.height, win.width)
        ev = None
        if events is not None:
            stream = torch.cuda.current_stream()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
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


def _box_union(boxes):
    """The bounding box (col0, row0, col1, row1) of boxes, or None for none."""
    boxes = [b for b in boxes if b is not None]
    if not boxes:
        return None
    return (min(b[0] for b in boxes), min(b[1] for b in boxes), max(b[2] for b in boxes),
            max(b[3] for b in boxes))


def _box_meet(a, b):
    if a is None or b is None:
        return None
    box = (max(a[0], b[0]), max(a[1], b[1]), min(a[2], b[2]), min(a[3], b[3]))
    return box if box[0] < box[2] and box[1] < box[3] else None


def _box_of(w: Window, grid: GridSpec):
    return _box_meet((w.col0, w.row0, w.col0 + w.width, w.row0 + w.height),
                     (0, 0, grid.width, grid.height))


class RankChain(PatchChain):
    """The chain with one patch per rank: rank k holds patch k and runs link k, the links in
    turn along the ranks. The only exchange is the halo each link needs from the chain so far:
    rank k - 1 sends rank k the chain's heights after link k - 1 over `halo(k)`, a box holding
    every cell an earlier patch covers that links k and later read (their lattices and windows),
    and rank k sends on the same for rank k + 1 after its own link (SourceChain::Seam,
    source_chain.cpp:144-152, with the prefix held where it was computed). Transfers are
    torch.distributed send / recv of one float32 box (NCCL over NVLink between GPUs, gloo on the
    host), so a link's solve never reads another rank's memory.

    compose(patch) returns this rank's share of the chain's heights: a mask of the cells its
    link gave data (for rank 0, its patch's data) and the grid's heights; the shares of all ranks
    are disjoint and together are PatchChain.compose's heights, bit for bit.
    """

    def __init__(self, device, grid: GridSpec, windows: list, seams: Seams, ranks,
                 tensors: str = "cuda"):
        if len(windows) != ranks.world:
            raise ValueError("RankChain needs one window per rank")
        self.ranks = ranks
        links = [ranks.rank] if ranks.rank > 0 else []
        super().__init__(device, grid, windows, seams, tensors=tensors, links=links)

    def halo(self, k: int):
        """The box (col0, row0, col1, row1) of the chain's heights rank k receives: the cells of
        patches before k within the bounding box of links k..n-1's lattices and windows."""
        reads = []
        for j in range(k, len(self.windows)):
            win, _ = self.lattice(j)
            reads += [_box_of(win, self.grid), _box_of(self.windows[j], self.grid)]
        earlier = _box_union([_box_of(w, self.grid) for w in self.windows[:k]])
        return _box_meet(_box_union(reads), earlier)

    def compose(self, patch, events=None):
        import torch
        import torch.distributed as dist

        k = self.ranks.rank
        self.heights.fill_(float("nan"))
        self.solves = []
        if k == 0:
            self.heights[self.windows[0].slices()].copy_(patch)
            mine = ~torch.isnan(self.heights)
        else:
            box = self.halo(k)
            if box is not None:
                buf = torch.empty((box[3] - box[1], box[2] - box[0]), dtype=torch.float32,
                                  device=self.heights.device)
                dist.recv(buf, src=k - 1)
                self.heights[box[1]:box[3], box[0]:box[2]].copy_(buf)
            before = torch.isnan(self.heights)
            self.link(k, patch, events)
            mine = before & ~torch.isnan(self.heights)
        if k + 1 < self.ranks.world:
            box = self.halo(k + 1)
            if box is not None:
                dist.send(self.heights[box[1]:box[3], box[0]:box[2]].contiguous(), dst=k + 1)
        return mine, self.heights
