"""Shared test set-up: the `gpu` marker, paths, and the GPU/device fixtures."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through libtgb200.so)")


@pytest.fixture(scope="session")
def device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    from terraingen_b200 import Device
    from terraingen_b200.build import build

    build()
    dev = Device(0)
    yield dev
    dev.close()


@pytest.fixture(scope="session")
def noise_fixture():
    return dict(np.load(GOLDEN / "noise.npz"))


@pytest.fixture(scope="session")
def crater_fixture():
    return dict(np.load(GOLDEN / "craters.npz"))


def grid_of(row):
    from terraingen_b200 import GridSpec

    w, h, x0, y0, pixel = row
    return GridSpec(int(w), int(h), float(x0), float(y0), float(pixel))
