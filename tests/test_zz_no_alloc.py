"""The allocation-free boulder bake (tg_boulders_bake_static), for callers that must not allocate
GPU memory mid-evaluation (a renderer's frame thread, a host with a fixed GPU memory budget),
against the allocating entry point (tg_boulders_bake) on the same inputs.

Collected last on purpose: the static form shares one scratch array across calls, and this file
checks that two calls in a row, after whatever ran before, give the allocating form's bits. Both
forms run the same count, scan, scatter and bake kernels on the same inputs, and the bake is a
max-composite (order-free), so their heights are identical, not merely close."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN, grid_of

pytestmark = pytest.mark.gpu


def bake_static(lib, boulders, grid, heights, width):
    """Calls tg_boulders_bake_static on device tensors; returns (status, message)."""
    import torch

    from terraingen_b200 import _native as N

    err = C.create_string_buffer(256)
    g = grid.native()
    handle = torch.cuda.current_stream().cuda_stream or 1  # torch's default stream: legacy
    status = lib.tg_boulders_bake_static(
        C.c_void_p(boulders.data_ptr()), boulders.numel() // 5, width, C.byref(g),
        C.c_void_p(heights.data_ptr()), N.NoData(0, 0.0), C.c_void_p(handle), err, 256)
    return status, err.value.decode()


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
        status, message = bake_static(lib, dev_b, grid, dev_h, grid.pixel)
        assert status == 0, message
        torch.cuda.synchronize()
        got = dev_h.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), name
        assert np.abs(got.astype(np.float64) - fx[f"{name}_expected"]).max() <= 1e-3
        assert np.count_nonzero(got != fx[f"{name}_base"]) > 1000


def test_static_bake_allocates_nothing(device):
    # A warm call leaves the device's free memory exactly as it was: no allocation by the
    # library, the CUDA runtime or torch (the inputs are allocated before the measurement).
    import torch

    from terraingen_b200 import library

    lib = library()
    fx = dict(np.load(GOLDEN / "boulders.npz"))
    grid = grid_of(fx["dense_grid"])
    dev_b = torch.from_numpy(np.ascontiguousarray(fx["dense_boulders"])).cuda()
    dev_h = torch.from_numpy(fx["dense_base"].copy()).cuda()
    assert bake_static(lib, dev_b, grid, dev_h, grid.pixel)[0] == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert bake_static(lib, dev_b, grid, dev_h, grid.pixel)[0] == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


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


def test_static_bake_entry_overflow_leaves_heights(device):
    # 13 boulders each covering a 4096^2 grid (128 x 128 bins): 212,992 binned entries, past the
    # scratch's 196,608. The call refuses with TG_ERROR_MEMORY before writing anything.
    import torch

    from terraingen_b200 import library
    from terraingen_b200.device import centered

    lib = library()
    grid = centered(4096, 4096, 1.0)
    stones = np.zeros((13, 5), np.float64)
    stones[:, 0] = np.linspace(-10.0, 10.0, 13)
    stones[:, 2] = 5000.0  # diameter: the dome's box covers the whole grid
    stones[:, 3] = 1.0
    stones[:, 4] = 1.0
    dev_b = torch.from_numpy(stones).cuda()
    base = torch.linspace(-1.0, 1.0, 4096 * 4096, dtype=torch.float32, device="cuda")
    dev_h = base.clone().reshape(4096, 4096)
    status, message = bake_static(lib, dev_b, grid, dev_h, 1.0)
    assert status == 4 and "196608" in message, (status, message)
    torch.cuda.synchronize()
    assert torch.equal(dev_h.reshape(-1), base)
    # The scratch is still good for the next call.
    fx = dict(np.load(GOLDEN / "boulders.npz"))
    g = grid_of(fx["fine_grid"])
    want = fx["fine_base"].copy()
    device.boulders_bake(np.ascontiguousarray(fx["fine_boulders"]), g, want, width=g.pixel)
    fine_h = torch.from_numpy(fx["fine_base"].copy()).cuda()
    status, message = bake_static(lib, torch.from_numpy(fx["fine_boulders"]).cuda(), g, fine_h,
                                  g.pixel)
    assert status == 0, message
    torch.cuda.synchronize()
    assert np.array_equal(fine_h.cpu().numpy().view(np.uint32), want.view(np.uint32))
