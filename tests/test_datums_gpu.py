"""GPU tests of crater datums (tg_crater_datums): the relief of older craters under each fitted
crater's plane-datum footprint, against the reference's own KernelDatumRelief on the inputs the
reference hands its GPU backend (tests/golden/datums.npz), and through the reference pipeline
with the drop-in device."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, grid_of
from oracle import harness as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def z():
    return dict(np.load(GOLDEN / "datums.npz"))


def _call(z):
    width, rows, first = (int(v) for v in z["call_shape"])
    return dict(kernel=z["call_kernel"], records=z["call_records"],
                data=z["call_data"].view(np.float32),
                band_floats=z["call_band_floats"].view(np.float32),
                band_cells=z["call_band_cells"].view(np.uint32),
                cells=z["call_cells"].view(np.uint32), entries=z["call_entries"].view(np.uint32),
                targets=z["call_targets"].view(np.uint32), width=width, rows=rows,
                first_row=first)


def test_datum_relief_matches_reference(device, z):
    c = _call(z)
    heights = z["call_heights"].view(np.float32).copy()
    before = heights.copy()
    device.crater_datums(c["kernel"], c["records"], c["data"], c["band_floats"],
                         c["band_cells"], c["cells"], c["entries"], c["targets"], heights,
                         c["width"], c["rows"], c["first_row"])
    want = z["relief"]
    changed = np.count_nonzero(want != before)
    assert changed > 1000
    assert np.array_equal(np.isnan(heights), np.isnan(want))
    ok = ~np.isnan(want)
    err = np.abs(heights[ok].astype(np.float64) - want[ok])
    # Float sums of profile heights; CUDA's powf / expf against the host's differ by an ulp.
    assert err.max() <= 1e-4, err.max()


def test_datum_relief_device_memory(device, z):
    import torch

    c = _call(z)
    host = z["call_heights"].view(np.float32).copy()
    device.crater_datums(c["kernel"], c["records"], c["data"], c["band_floats"],
                         c["band_cells"], c["cells"], c["entries"], c["targets"], host,
                         c["width"], c["rows"], c["first_row"])
    t = {k: torch.from_numpy(np.ascontiguousarray(c[k])).cuda()
         for k in ("records", "data", "band_floats", "cells", "entries")}
    t["kernel"] = c["kernel"]  # the parameter block stays on the host
    t["band_cells"] = torch.from_numpy(c["band_cells"].view(np.int32)).cuda()
    t["targets"] = torch.from_numpy(c["targets"].view(np.int32)).cuda()
    heights = torch.from_numpy(z["call_heights"].view(np.float32).copy()).cuda()
    device.crater_datums(t["kernel"], t["records"], t["data"], t["band_floats"], t["band_cells"],
                         t["cells"].view(torch.int32), t["entries"].view(torch.int32),
                         t["targets"], heights, c["width"], c["rows"], c["first_row"])
    torch.cuda.synchronize()
    assert np.array_equal(heights.cpu().numpy().view(np.uint32), host.view(np.uint32))


def test_datum_scene_through_reference_pipeline(device, z):
    # Terrain::Evaluate with Backend::Cuda: the adapter runs the datum relief on tg_crater_datums
    # and the ordered datum craters on tg_craters_apply_lists.
    if not H.available("libtgref_cuda.so"):
        pytest.skip("oracle/_ref/libtgref_cuda.so was not built with the reference")
    import sys

    sys.path.insert(0, str(GOLDEN))
    from make_fixtures import DATUM_SCENE

    _, fields = DATUM_SCENE
    from terraingen_b200.layouts import FRACTAL

    src = z["source"].view(FRACTAL)
    scene = H.make_scene(grid_of(z["grid"]), source_fractals=src, craters=fields)
    gpu, _ = H.evaluate(H.dropin(), scene, 1, 1)
    want = z["expected"]
    err = np.abs(gpu.astype(np.float64) - want)
    assert err.max() <= 1e-3, err.max()


def test_datum_relief_refuses_a_bad_index(device, z):
    from terraingen_b200 import TgError

    c = _call(z)
    targets = c["targets"].copy()
    targets[0] = 10 ** 6  # no such record
    heights = z["call_heights"].view(np.float32).copy()
    with pytest.raises(TgError):
        device.crater_datums(c["kernel"], c["records"], c["data"], c["band_floats"],
                             c["band_cells"], c["cells"], c["entries"], targets, heights,
                             c["width"], c["rows"], c["first_row"])
