"""The allocation-free boulder bake (tg_boulders_bake_static), for callers that must not allocate
GPU memory mid-evaluation (a renderer's frame thread, a host with a fixed GPU memory budget),
against the allocating entry point (tg_boulders_bake) on the same inputs.

Collected last on purpose: the static form shares one scratch array across calls, and this file
checks that two calls in a row, after whatever ran before, agree with the allocating form."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN, grid_of

pytestmark = pytest.mark.gpu

TOLERANCE_M = 1e-3


def bake_static(lib, boulders, grid, heights, width):
    import torch

    from terraingen_b200 import _native as N

    err = C.create_string_buffer(256)
    g = grid.native()
    handle = torch.cuda.current_stream().cuda_stream or 1  # torch's default stream: legacy
    status = lib.tg_boulders_bake_static(
        C.c_void_p(boulders.data_ptr()), boulders.numel() // 5, width, C.byref(g),
        C.c_void_p(heights.data_ptr()), N.NoData(0, 0.0), C.c_void_p(handle), err, 256)
    assert status == 0, err.value.decode()


@pytest.mark.parametrize("first,second", [("dense", "fine"), ("fine", "dense")])
def test_static_bake_matches_allocating_bake_twice(device, first, second):
    import torch

    from terraingen_b200 import library

    lib = library()
    fx = dict(np.load(GOLDEN / "boulders.npz"))
    for name in (first, second):
        grid = grid_of(fx[f"{name}_grid"])
        boulders = np.ascontiguousarray(fx[f"{name}_boulders"])
        want = fx[f"{name}_base"].copy()
        device.boulders_bake(boulders, grid, want, width=grid.pixel)
        dev_b = torch.from_numpy(boulders).cuda()
        dev_h = torch.from_numpy(fx[f"{name}_base"].copy()).cuda()
        bake_static(lib, dev_b, grid, dev_h, grid.pixel)
        torch.cuda.synchronize()
        got = dev_h.cpu().numpy()
        err = np.abs(got.astype(np.float64) - want)
        assert err.max() <= TOLERANCE_M, (name, err.max())
        assert np.count_nonzero(got != fx[f"{name}_base"]) > 1000


def test_static_bake_refuses_oversize(device):
    import torch

    from terraingen_b200 import GridSpec, _native as N, library

    lib = library()
    grid = GridSpec(8, 8, 0.0, 8.0, 1.0)
    boulders = torch.zeros((70000, 5), dtype=torch.float64, device="cuda")
    heights = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    err = C.create_string_buffer(256)
    g = grid.native()
    status = lib.tg_boulders_bake_static(C.c_void_p(boulders.data_ptr()), 70000, 1.0, C.byref(g),
                                         C.c_void_p(heights.data_ptr()), N.NoData(0, 0.0),
                                         C.c_void_p(1), err, 256)
    assert status == 1 and b"65536" in err.value
