"""Crater batches with their records made on the device (tg_crater_batch_device) against the host
builder (tg_crater_batch, itself bit-exact with the reference's MakeCraterKernelBatch: see
tests/test_population.py): kernel, records, data and footprints byte for byte, on the synthetic
terrain's whole tile and on scenes with every profile, outlines on and off, wall terraces and
massif peaks; sizes, capacities and the empty batch."""
from __future__ import annotations

import numpy as np
import pytest

from terraingen_b200 import _native as N
from terraingen_b200.device import centered
from terraingen_b200.layouts import CRATER_RECORD
from terraingen_b200.workloads import config2_shaping, crater_batch, crater_population

pytestmark = pytest.mark.gpu


def _terrain_population():
    full_area = (4097 * 0.5) ** 2
    return crater_population(7, 200000.0 / (full_area * (1.0 ** -2.0 - 500.0 ** -2.0)), 1.0, 500.0)


def _terraced_population():
    return N.Population(seed=9, sfd_coefficient=0.6, sfd_exponent=2.0, min_diameter=8.0,
                        max_diameter=300.0, lifetime_gyr=1.0, depth_ratio=0.2, rim_ratio=0.04,
                        cutoff_depth_ratio=0.04, cell_size_factor=16.0, margin_radii=0.0,
                        min_resolved_diameter=0.0)


SCENES = {
    "terrain4097": (_terrain_population, config2_shaping, lambda: centered(4097, 4097, 0.5)),
    "ft_plain": (lambda: crater_population(3, 0.02, 1.0, 200.0),
                 lambda: N.Shaping(profile=0, irregular=0), lambda: centered(700, 500, 0.5,
                                                                             1.0e4, -3.0e3)),
    "mpd_outlines": (lambda: crater_population(5, 0.02, 1.0, 200.0),
                     lambda: N.Shaping(profile=1, irregular=1), lambda: centered(640, 640, 0.5)),
    "terraced_peaked": (_terraced_population,
                        lambda: N.Shaping(profile=2, irregular=1, transition_diameter=60.0,
                                          terrace_onset=80.0, terrace_full=200.0,
                                          terrace_min_freshness=0.3),
                        lambda: centered(192, 192, 2.0)),
}


def _device_batch(device, pop, shaping, grid):
    import torch

    _, nr, nd = device.crater_batch(pop, shaping, grid)
    records = torch.empty(max(nr, 1) * CRATER_RECORD.itemsize, dtype=torch.uint8, device="cuda")
    data = torch.empty(max(nd, 1), dtype=torch.float32, device="cuda")
    foot = torch.empty(3 * max(nr, 1), dtype=torch.float64, device="cuda")
    kernel, nr2, nd2 = device.crater_batch(pop, shaping, grid, records, data, foot)
    torch.cuda.synchronize()
    assert (nr2, nd2) == (nr, nd)
    return (kernel, records.cpu().numpy()[:nr * CRATER_RECORD.itemsize], data.cpu().numpy()[:nd],
            foot.cpu().numpy()[:3 * nr])


@pytest.mark.parametrize("name", sorted(SCENES))
def test_device_records_are_the_host_batch(device, name):
    make_pop, make_shaping, make_grid = SCENES[name]
    pop, shaping, grid = make_pop(), make_shaping(), make_grid()
    kernel, records, data, foot = crater_batch(pop, grid, shaping=shaping)
    assert len(records) > 50
    if name == "terraced_peaked":
        assert np.count_nonzero(records["terraceCount"]) > 0
        assert np.count_nonzero(records["peakCount"]) > 0
    got = _device_batch(device, pop, shaping, grid)
    assert got[0].tobytes() == kernel.tobytes()
    want = records.view(np.uint8).ravel()
    if not np.array_equal(got[1], want):
        rows = np.nonzero((got[1].reshape(-1, 144) != want.reshape(-1, 144)).any(axis=1))[0]
        first = got[1].reshape(-1, 144)[rows[0]].view(CRATER_RECORD)[0]
        raise AssertionError(f"{len(rows)} records differ, first {rows[0]}: {first} against "
                             f"{records[rows[0]]}")
    assert np.array_equal(got[2].view(np.uint32), data.view(np.uint32))
    assert np.array_equal(got[3].view(np.uint64), foot.view(np.uint64))


def test_device_records_twice_and_capacity(device):
    import torch

    pop, shaping, grid = crater_population(3, 0.02, 1.0, 200.0), N.Shaping(profile=0,
                                                                             irregular=1), \
        centered(512, 512, 0.5)
    first = _device_batch(device, pop, shaping, grid)
    again = _device_batch(device, pop, shaping, grid)
    assert all(np.array_equal(a, b) for a, b in zip(first[1:], again[1:]))
    _, nr, nd = device.crater_batch(pop, shaping, grid)
    small = torch.empty((nr - 1) * CRATER_RECORD.itemsize, dtype=torch.uint8, device="cuda")
    data = torch.empty(nd, dtype=torch.float32, device="cuda")
    with pytest.raises(N.TgError) as error:
        device.crater_batch(pop, shaping, grid, small, data, None)
    assert error.value.status == 1  # TG_ERROR_ARGUMENT


def test_device_records_empty_batch(device):
    import torch

    # Every crater below two samples across: no record, and the one data float 0.
    pop, shaping, grid = crater_population(3, 0.02, 0.1, 0.9), N.Shaping(profile=0, irregular=1), \
        centered(256, 256, 0.5)
    kernel, records, data, foot = crater_batch(pop, grid, shaping=shaping)
    assert len(records) == 0 and len(data) == 1
    out = torch.full((1,), 7.0, dtype=torch.float32, device="cuda")
    got, nr, nd = device.crater_batch(pop, shaping, grid, None, out, None)
    torch.cuda.synchronize()
    assert (nr, nd) == (0, 1) and float(out[0]) == 0.0
    assert got.tobytes() == kernel.tobytes()


def test_evaluate_with_device_records_equals_host_records(device):
    # The e2e path: the batch made on the device and evaluated in device memory gives the heights
    # of the host-built batch evaluated with host buffers, bit for bit.
    import torch

    from terraingen_b200.layouts import fractal
    from terraingen_b200.workloads import boulder_population, generate_boulders

    grid = centered(1025, 769, 0.5, 120.0, -40.0)
    pop, shaping = _terrain_population(), config2_shaping()
    fractals = np.array([fractal(seed=7, wavelength=512.0, amplitude=5.0, octaves=8)])
    full_area = (4097 * 0.5) ** 2
    stones = generate_boulders(boulder_population(7, 1e6 / (full_area * (0.2 ** -2.5 -
                                                                          3.0 ** -2.5))), grid)
    kernel, records, data, foot = crater_batch(pop, grid, shaping=shaping)
    want = np.zeros((grid.height, grid.width), np.float32)
    device.evaluate(grid, want, fractals=fractals, craters=(kernel, records, data, foot),
                    boulders=stones, boulder_width=0.5)
    got_kernel, rec_d, data_d, foot_d = _device_batch(device, pop, shaping, grid)
    cuda = dict(device="cuda")
    heights = torch.empty((grid.height, grid.width), dtype=torch.float32, **cuda)
    device.evaluate(grid, heights, fractals=fractals,
                    craters=(got_kernel, torch.from_numpy(rec_d).to(**cuda),
                             torch.from_numpy(data_d).to(**cuda),
                             torch.from_numpy(foot_d).to(**cuda)),
                    boulders=torch.from_numpy(np.ascontiguousarray(stones).ravel()).to(**cuda),
                    boulder_width=0.5)
    torch.cuda.synchronize()
    assert np.array_equal(heights.cpu().numpy().view(np.uint32), want.view(np.uint32))
