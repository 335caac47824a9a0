"""Test configuration: the `gpu` marker, import paths and shared helpers.

CPU tests (``-m "not gpu"``) pin the oracle against the golden fixtures and the
compiled reference, check the host logic and that the C-ABI library loads and
exports every function of include/octree_b200.h.  GPU tests (``-m gpu``) are
the parity tests of the CUDA path against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the device library")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port, build_port

    build_port()
    return Port()
