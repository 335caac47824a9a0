"""The C++ drop-in (include/linear_octree_gpu.hpp): compile tests/cpp/test_wrapper.cpp
with g++ against the header and liboctree_b200.so, then run it on the GPU.  The
program restates the reference's GoogleTest cases through the C++ API."""
import os
import shutil
import subprocess

import pytest

from octrees_benchmark_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_wrapper_test(out_dir):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = os.path.join(out_dir, "test_wrapper")
    libdir = os.path.dirname(capi.LIB_PATH)
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "test_wrapper.cpp"), "-o", exe, "-L", libdir, "-loctree_b200",
           "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True)
    return exe


def test_wrapper_compiles(tmp_path):
    capi.lib()  # the library must exist (fails loudly otherwise)
    assert os.path.exists(compile_wrapper_test(str(tmp_path)))


@pytest.mark.gpu
def test_wrapper_reference_cases_on_gpu(tmp_path):
    exe = compile_wrapper_test(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
