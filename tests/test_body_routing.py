"""The adapter's routing on a body, without a GPU: the reference pipeline (Backend::Cuda on the
capture build of the adapter, oracle/_ref/libtgref_capture.so) dispatches its crater kernel on a
sphere with tiles[2] == 1, and the adapter hands it to tg_craters_apply_body (capture kind 4) with
a 52-byte frame per record and a 24-byte split point per cell."""

from __future__ import annotations

import ctypes as C
import importlib.util

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import harness as H


def test_body_craters_go_to_the_body_entry_point():
    if not H.available("libtgref_capture.so"):
        pytest.skip("oracle/_ref/libtgref_capture.so was not built with the reference")
    spec = importlib.util.spec_from_file_location("body_cases", GOLDEN / "body_cases.py")
    cases = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cases)
    lib = H.capture()
    before = lib.tgref_capture_count()
    scene = cases.scene()
    out = np.zeros(scene.width * scene.height, np.float32)
    assert lib.tgref_evaluate(C.byref(scene), 1, 1, out.ctypes.data, C.byref(C.c_double())) == 0
    info = np.zeros(8, np.uint32)
    kinds = []
    for i in range(before, lib.tgref_capture_count()):
        lib.tgref_capture_info(i, info.ctypes.data)
        kinds.append(int(info[0]))
        if info[0] == 4:
            assert (info[1], info[2]) == (scene.width, scene.height)
    assert kinds == [4]


def test_body_datums_go_to_the_body_datum_entry_point():
    if not H.available("libtgref_capture.so"):
        pytest.skip("oracle/_ref/libtgref_capture.so was not built with the reference")
    spec = importlib.util.spec_from_file_location("body_cases", GOLDEN / "body_cases.py")
    cases = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cases)
    lib = H.capture()
    before = lib.tgref_capture_count()
    scene = cases.scene(datum=1)
    out = np.zeros(scene.width * scene.height, np.float32)
    assert lib.tgref_evaluate(C.byref(scene), 1, 1, out.ctypes.data, C.byref(C.c_double())) == 0
    info = np.zeros(8, np.uint32)
    kinds = []
    for i in range(before, lib.tgref_capture_count()):
        lib.tgref_capture_info(i, info.ctypes.data)
        kinds.append(int(info[0]))
    assert kinds == [5, 4]
