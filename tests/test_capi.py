"""CPU checks of the C-ABI library: it loads, exports every function that
include/octree_b200.h declares, and its host-only logic behaves (no kernel is
launched here)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import octrees_benchmark_b200 as ob
from octrees_benchmark_b200 import capi
from tests.conftest import HAS_GPU


def test_library_exports_every_header_function():
    L = ob.lib()
    names = ob.header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the binding covers the whole header
    assert sorted(capi.SIGNATURES) == names


def test_library_dynamic_symbols_match_header():
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln and ln.split()[-1].startswith("oct_")}
    assert exported == set(ob.header_functions())


def test_status_strings_and_version():
    L = ob.lib()
    assert L.oct_abi_version() == 1
    assert L.oct_status_string(capi.OCT_OK) == b"ok"
    assert L.oct_status_string(capi.OCT_ERR_CAPACITY) == b"output capacity too small"
    assert L.oct_status_string(999) == b"unknown status"


def test_null_and_bad_arguments_are_rejected_without_a_device():
    L = ob.lib()
    h = C.c_void_p()
    assert L.oct_cloud_create(None, C.byref(h)) == capi.OCT_ERR_INVALID_ARG
    bad = capi.OctParams(128, 3, 0, 0)  # encoder 3 is a 2D encoder: not usable by the octree
    assert L.oct_cloud_create(C.byref(bad), C.byref(h)) == capi.OCT_ERR_INVALID_ARG
    assert L.oct_cloud_destroy(None) == capi.OCT_ERR_INVALID_ARG
    assert L.oct_build(None, None) == capi.OCT_ERR_INVALID_ARG
    assert L.oct_knn(None, None, 0, 1, None, None, None, 0) == capi.OCT_ERR_INVALID_ARG


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device status")
def test_create_without_device_reports_no_device():
    L = ob.lib()
    h = C.c_void_p()
    p = capi.OctParams(128, 5, 0, 0)
    assert L.oct_cloud_create(C.byref(p), C.byref(h)) == capi.OCT_ERR_NO_DEVICE
    assert not h.value
    with pytest.raises(capi.OctError) as ei:
        ob.LinearOctree(np.zeros((4, 3)))
    assert ei.value.status == capi.OCT_ERR_NO_DEVICE


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(capi, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(capi, "_lib", None)
    with pytest.raises(ImportError):
        capi.lib()
