"""One process per GPU: the rank plumbing the benchmark's multi-GPU runs share.

The evaluation path shards without exchange: each rank evaluates its own tiles, uneven tiles,
request stream or DEM refinement (weak scaling), and only timings cross ranks, reduced to their
maximum. `setup` reads the torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_*); the
backend is NCCL on GPUs and gloo for the CPU tests of this module.
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local: int
    device: str  # "cuda" or "cpu": where reductions run


def setup(backend: str = "nccl", timeout_s: float = 300.0) -> Ranks:
    """The process's rank; joins the process group when the world has more than one rank."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    device = "cuda" if backend == "nccl" else "cpu"
    if world > 1:
        import torch
        import torch.distributed as dist

        kwargs = {}
        if device == "cuda":
            torch.cuda.set_device(local)
            kwargs["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kwargs)
    return Ranks(rank, world, local, device)


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, r: Ranks) -> float:
    """The largest of every rank's `value` (timings: the slowest rank bounds the job)."""
    if r.world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=r.device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_floats(values: list, r: Ranks) -> list:
    """Every rank's list of floats (same length on each), rank by rank."""
    if r.world == 1:
        return [list(values)]
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=r.device)
    out = [torch.zeros_like(t) for _ in range(r.world)]
    dist.all_gather(out, t)
    return [o.tolist() for o in out]


def teardown(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# The benchmark's per-rank workloads: disjoint in space or seed, the same size on every rank.
def terrain_center(rank: int, side: int = 4097, pixel: float = 0.5) -> tuple:
    """Rank `rank`'s 4097^2 tile center: tiles side by side along x."""
    return (rank * side * pixel, 0.0)


def tiles_seed(rank: int) -> int:
    return 11 + 7919 * rank


def stream_seeds(rank: int) -> tuple:
    """Warm-up, real-time and saturated request stream seeds."""
    return (1 + rank, 2 + rank, 3 + rank)


def dem_seed(rank: int) -> int:
    return 7 + 10 * rank
