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
