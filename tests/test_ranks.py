"""The multi-rank plumbing on CPU: world size 2 over gloo, 127.0.0.1 rendezvous.

Each rank joins, reduces its timing to the maximum over ranks, gathers every rank's workload
identity, and checks the shards the benchmark gives them are disjoint (different tile places,
tile sets, request streams and DEM seeds) and the same size.
"""

from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, queue) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from terraingen_b200 import ranks
    from terraingen_b200.workloads import uneven_tiles

    r = ranks.setup("gloo", timeout_s=60.0)
    try:
        assert (r.rank, r.world) == (rank, world)
        slowest = ranks.max_over_ranks(1.0 + rank, r)
        ts = uneven_tiles(6, seed=ranks.tiles_seed(rank), boulders=False)
        ident = [ranks.terrain_center(rank)[0], float(ranks.tiles_seed(rank)),
                 float(ts.cells), float(ranks.dem_seed(rank)), float(ranks.stream_seeds(rank)[2]),
                 float(ts.grids[0].x0)]
        everyone = ranks.gather_floats(ident, r)
        ranks.barrier(r)
        queue.put((rank, slowest, everyone))
    finally:
        ranks.teardown(r)


def test_two_ranks_over_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(k, 2, port, queue)) for k in range(2)]
    for p in procs:
        p.start()
    results = dict((rank, (slowest, everyone)) for rank, slowest, everyone in
                   (queue.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        slowest, everyone = results[rank]
        assert slowest == 2.0  # the maximum over ranks, on both
        a, b = everyone
        assert a[0] != b[0] and a[1] != b[1] and a[3] != b[3] and a[4] != b[4]
        assert a[5] != b[5]  # different tile sets
    assert results[0][1] == results[1][1]


def test_single_rank_needs_no_group(monkeypatch):
    from terraingen_b200 import ranks

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    r = ranks.setup("gloo")
    assert (r.rank, r.world) == (0, 1)
    assert ranks.max_over_ranks(3.5, r) == 3.5
    assert ranks.gather_floats([1.0, 2.0], r) == [[1.0, 2.0]]


class _HostSeams:
    """A host stand-in for the device's seam calls, deterministic and with the real calls' data
    dependencies: samples read both rasters on the lattice, the solve smooths the differences
    over the lattice, the fill writes the later raster plus the field into the window's gaps. It
    checks how RankChain moves the chain between ranks, not the seam arithmetic (the GPU tests do
    that)."""

    def seam_samples(self, earlier, later, grid, col0, row0, lw, lh, data, difference):
        import torch

        e = torch.full((lh, lw), float("nan"))
        lt = torch.full((lh, lw), float("nan"))
        r0, r1 = max(row0, 0), min(row0 + lh, grid.height)
        c0, c1 = max(col0, 0), min(col0 + lw, grid.width)
        e[r0 - row0:r1 - row0, c0 - col0:c1 - col0] = earlier[r0:r1, c0:c1]
        lt[r0 - row0:r1 - row0, c0 - col0:c1 - col0] = later[r0:r1, c0:c1]
        data.copy_((~torch.isnan(e)).to(torch.uint8) + 2 * (~torch.isnan(lt)).to(torch.uint8))
        difference.copy_(torch.nan_to_num(e - lt, nan=0.0))

    def seam_solve(self, data, difference, dx, dy, mode, field, **kwargs):
        import torch

        f = torch.where(data == 3, difference, torch.zeros_like(difference))
        for _ in range(3):
            g = f.clone()
            g[1:-1, 1:-1] = 0.25 * (f[:-2, 1:-1] + f[2:, 1:-1] + f[1:-1, :-2] + f[1:-1, 2:])
            f = torch.where(data == 3, f, g)
        field.copy_(f)
        return field, {"iterations": 3}

    def seam_fill(self, field, lattice, later, grid, heights, window):
        import torch

        col0, row0, w, h = window
        lc0 = round((lattice.x0 - grid.x0) / grid.pixel)
        lr0 = round((grid.y0 - lattice.y0) / grid.pixel)
        f = torch.zeros((h, w))
        r0, r1 = max(row0, lr0), min(row0 + h, lr0 + field.shape[0])
        c0, c1 = max(col0, lc0), min(col0 + w, lc0 + field.shape[1])
        if r0 < r1 and c0 < c1:
            f[r0 - row0:r1 - row0, c0 - col0:c1 - col0] = field[r0 - lr0:r1 - lr0, c0 - lc0:c1 - lc0]
        out = heights[row0:row0 + h, col0:col0 + w]
        src = later[row0:row0 + h, col0:col0 + w] + f
        gaps = torch.isnan(out) & ~torch.isnan(src)
        out[gaps] = src[gaps]


def _chain_case(world: int):
    """A grid, `world` overlapping windows (in a row for 2, a 2 x 2 layout for 4) and patches."""
    import torch

    from terraingen_b200.chain import Seams, Window
    from terraingen_b200.device import GridSpec

    grid = GridSpec(96, 80, 0.0, 80.0, 1.0)
    if world == 2:
        windows = [Window(0, 0, 56, 80), Window(40, 0, 56, 80)]
    else:
        windows = [Window(0, 0, 52, 44), Window(44, 0, 52, 44), Window(0, 36, 52, 44),
                   Window(44, 36, 52, 44)]
    g = torch.Generator().manual_seed(5)
    patches = []
    for w in windows:
        p = torch.randn((w.height, w.width), generator=g)
        p[torch.rand((w.height, w.width), generator=g) < 0.05] = float("nan")  # holes
        patches.append(p)
    return grid, windows, Seams(mode="height", decay_length=2.0), patches


def _chain_rank(rank: int, world: int, port: int, queue) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from terraingen_b200 import ranks
    from terraingen_b200.chain import RankChain

    r = ranks.setup("gloo", timeout_s=60.0)
    try:
        grid, windows, seams, patches = _chain_case(world)
        chain = RankChain(_HostSeams(), grid, windows, seams, r, tensors="cpu")
        mine, heights = chain.compose(patches[rank])
        queue.put((rank, mine.numpy().copy(), heights.numpy().copy()))
        ranks.barrier(r)
    finally:
        ranks.teardown(r)


@pytest.mark.parametrize("world", [2, 4])
def test_rank_chain_matches_single_rank_chain(world):
    # The seam chain split one patch per rank (gloo ranks on the host) gives the single-rank
    # chain's heights bit for bit: each rank's share (the cells its link filled) is disjoint
    # from the others' and together they are the whole chain.
    import numpy as np
    import torch.multiprocessing as mp

    from terraingen_b200.chain import PatchChain

    grid, windows, seams, patches = _chain_case(world)
    want = PatchChain(_HostSeams(), grid, windows, seams, tensors="cpu").compose(patches).numpy()
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_chain_rank, args=(k, world, port, queue)) for k in range(world)]
    for p in procs:
        p.start()
    shares = dict((rank, (mine, heights)) for rank, mine, heights in
                  (queue.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.full(want.shape, np.nan, np.float32)
    covered = np.zeros(want.shape, bool)
    for rank in range(world):
        mine, heights = shares[rank]
        assert not np.any(covered & mine)  # disjoint shares
        got[mine] = heights[mine]
        covered |= mine
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.array_equal(got[~np.isnan(got)].view(np.uint32), want[~np.isnan(want)].view(np.uint32))
    assert covered.sum() > 0.9 * want.size
