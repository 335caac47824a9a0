"""The allocation-free entry point oct_encode_sort_noalloc.

Some callers cannot allocate device memory when they call in: code that runs
inside a memory pool it does not own, plugin hosts that forbid cudaMalloc and
cudaFree on their streams, and latency-bound loops that cannot afford the
device-wide synchronisation an allocation causes.  For them the library keeps
its sort scratch in one fixed device array and the caller passes only the
points and the outputs.  This test calls that entry point through the C ABI,
three times in a row on one stream (different clouds, large after small and
small after large, so each call runs on scratch the previous call left
behind) and once on an empty cloud, and checks each result bit for bit
against the regular entry point oct_encode_sort.  It lives in a file of its
own that pytest collects last, and it passes both alone in a fresh process and
after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from octrees_benchmark_b200 import capi
from octrees_benchmark_b200.synth import lidar_tile
from tests.parity import same_f64

pytestmark = pytest.mark.gpu


def regular_encode_sort(xyz, encoder):
    """Keys, ids and Box from the regular (allocating) entry point, host buffers."""
    L = capi.lib()
    p = capi.OctParams(64, encoder, 0, 0)
    h = C.c_void_p()
    capi.check(L.oct_cloud_create(C.byref(p), C.byref(h)), None, "create")
    try:
        n = len(xyz)
        capi.check(L.oct_set_points(h, xyz.ctypes.data, n, 0), h)
        box = np.zeros(12)
        keys = np.zeros(n, np.uint64)
        perm = np.zeros(n, np.uint32)
        capi.check(L.oct_encode_sort(h, box.ctypes.data, keys.ctypes.data, perm.ctypes.data, None, 0), h)
        return keys, perm, box
    finally:
        L.oct_cloud_destroy(h)


def test_noalloc_matches_regular_entry_point_on_calls_in_a_row():
    torch = pytest.importorskip("torch")
    L = capi.lib()
    # small after large too: the third call runs on scratch (look-back words beyond its own tiles) that the
    # largest cloud left behind
    clouds = [(lidar_tile(200_003, 220.0, seed=41), capi.ENCODERS["hilbert"]),
              (lidar_tile(capi.OCT_NOALLOC_MAX_POINTS, 240.0, seed=42), capi.ENCODERS["morton"]),
              (lidar_tile(5_000, 30.0, seed=44), capi.ENCODERS["hilbert"])]
    dev_in, dev_out = [], []
    for xyz, _ in clouds:
        n = len(xyz)
        dev_in.append(torch.from_numpy(np.ascontiguousarray(xyz)).cuda())
        dev_out.append((torch.empty(n, dtype=torch.int64, device="cuda"),
                        torch.empty(n, dtype=torch.int32, device="cuda"),
                        torch.empty(12, dtype=torch.float64, device="cuda")))
    torch.cuda.synchronize()
    # calls in a row on the default stream; each reuses the scratch the previous one left behind
    free_before_second = None
    for i, ((xyz, enc), d_xyz, (keys, perm, box)) in enumerate(zip(clouds, dev_in, dev_out)):
        if i == 1:
            torch.cuda.synchronize()
            free_before_second = torch.cuda.mem_get_info()[0]
        st = L.oct_encode_sort_noalloc(enc, d_xyz.data_ptr(), len(xyz), keys.data_ptr(), perm.data_ptr(),
                                       box.data_ptr(), None)
        assert st == capi.OCT_OK
    torch.cuda.synchronize()
    # the later calls allocated nothing on the device
    assert torch.cuda.mem_get_info()[0] == free_before_second
    for (xyz, enc), (keys, perm, box) in zip(clouds, dev_out):
        rk, rp, rb = regular_encode_sort(xyz, enc)
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), rk)
        assert np.array_equal(perm.cpu().numpy().view(np.uint32), rp)
        assert same_f64(box.cpu().numpy(), rb)
        assert np.all(box.cpu().numpy()[3:6] >= 0.0)  # -1.0 would flag a sort pass that gave up


def test_noalloc_empty_cloud_gives_the_regular_box():
    torch = pytest.importorskip("torch")
    L = capi.lib()
    box = torch.full((12,), 7.0, dtype=torch.float64, device="cuda")
    st = L.oct_encode_sort_noalloc(5, None, 0, None, None, box.data_ptr(), None)
    assert st == capi.OCT_OK
    torch.cuda.synchronize()
    _, _, rb = regular_encode_sort(np.zeros((0, 3)), 5)
    assert same_f64(box.cpu().numpy(), rb)


def test_noalloc_accepts_a_buffer_that_is_only_8_byte_aligned():
    torch = pytest.importorskip("torch")
    L = capi.lib()
    xyz = lidar_tile(30_001, 60.0, seed=43)
    flat = torch.zeros(3 * len(xyz) + 1, dtype=torch.float64, device="cuda")
    flat[1:] = torch.from_numpy(xyz.reshape(-1)).cuda()
    d_xyz = flat[1:]  # 8-byte offset from a 256-byte aligned allocation
    n = len(xyz)
    keys = torch.empty(n + 1, dtype=torch.int64, device="cuda")[1:]
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    box = torch.empty(12, dtype=torch.float64, device="cuda")
    st = L.oct_encode_sort_noalloc(5, d_xyz.data_ptr(), n, keys.data_ptr(), perm.data_ptr(), box.data_ptr(), None)
    assert st == capi.OCT_OK
    torch.cuda.synchronize()
    rk, rp, rb = regular_encode_sort(xyz, 5)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), rk)
    assert np.array_equal(perm.cpu().numpy().view(np.uint32), rp)
    assert same_f64(box.cpu().numpy(), rb)


def test_noalloc_rejects_clouds_above_the_limit():
    torch = pytest.importorskip("torch")
    L = capi.lib()
    n = capi.OCT_NOALLOC_MAX_POINTS + 1
    d_xyz = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    box = torch.empty(12, dtype=torch.float64, device="cuda")
    st = L.oct_encode_sort_noalloc(5, d_xyz.data_ptr(), n, keys.data_ptr(), perm.data_ptr(), box.data_ptr(), None)
    assert st == capi.OCT_ERR_INVALID_ARG
    # an encoder the octree cannot use is rejected too
    st = L.oct_encode_sort_noalloc(3, d_xyz.data_ptr(), 16, keys.data_ptr(), perm.data_ptr(), box.data_ptr(), None)
    assert st == capi.OCT_ERR_INVALID_ARG
