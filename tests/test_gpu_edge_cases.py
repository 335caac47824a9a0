"""Edge cases on the device, each checked against the oracle: the reference's
own GoogleTest cases (tests/structures/test_octree.cpp,
test_octree_advanced.cpp, tests/integration/test_complex.cpp) restated, and the
degenerate inputs the reference handles (empty cloud, one point, all points
equal, flat axes, huge offsets, leaf size 1, zero radius, queries outside the
box), plus the device-buffer form of the ABI and error statuses."""
import ctypes as C

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from tests.parity import assert_csr_equal, assert_knn_equal, assert_ranges_equal, same_f64, sq_dist

pytestmark = pytest.mark.gpu

KERNELS = {"sphere": 1, "circle": 0, "cube": 3, "square": 2}
ALGO_NAMES = {1: "neighbors", 2: "neighborsPrune", 3: "neighborsStruct"}


SEARCH_PATHS = [dict(packet=False, fp32_filter=False), dict(packet=True, fp32_filter=False),
                dict(packet=True, fp32_filter=True)]


def full_check(port, pts, enc=1, leaf=128, centers=None, radii=(0.0, 0.25, 1.0, 2.5), ks=(1, 2, 5)):
    for path in SEARCH_PATHS:
        oc, sxyz = full_check_path(port, pts, enc, leaf, centers, radii, ks, path)
    return oc, sxyz


def full_check_path(port, pts, enc, leaf, centers, radii, ks, path):
    pts = np.asarray(pts, np.float64).reshape(-1, 3)
    keys, perm, box, sxyz = port.encode_sort(enc, pts)
    t = port.build(enc, keys, leaf, box)
    oc = LinearOctree(pts, encoder=enc, max_points_leaf=leaf, **path)
    gk, gp, gx = oc.sorted_points()
    assert same_f64(oc.box, box)
    assert np.array_equal(gk, keys) and np.array_equal(gp, perm) and same_f64(gx, sxyz)
    assert (oc.n_leaf, oc.n_internal, oc.n_total, oc.max_depth_seen) == (t.n_leaf, t.n_internal, t.n_total,
                                                                          t.max_depth)
    ex, ax = oc.export(), t.arrays()
    assert np.array_equal(ex["offsets"], ax["offsets"]) and np.array_equal(ex["ranges"], ax["ranges"])
    for k in ("centers", "radii", "half"):
        assert same_f64(ex[k], ax[k]), k
    if centers is None:
        centers = np.concatenate([sxyz[: min(len(sxyz), 20)], np.zeros((1, 3)), np.full((1, 3), 1e3)])
    centers = np.asarray(centers, np.float64).reshape(-1, 3)
    for r in radii:
        for kn, kv in KERNELS.items():
            for algo in (1, 2, 3):
                offs, idx = oc.radius_search(centers, r, kn, ALGO_NAMES[algo])
                o2, i2 = t.radius(sxyz, kv, algo, centers, r)
                assert_csr_equal(offs, idx, o2, i2, f"{kn} {algo} r={r}")
            ro, pairs, _ = oc.neighborsStruct(centers, r, kn)
            o2, p2 = t.struct_ranges(sxyz, kv, centers, r)
            assert_ranges_equal(ro, pairs, o2, p2, kn)
    for k in ks:
        idx, d2, cnt = oc.knn(centers, k)
        i2, d22, c2 = t.knn(sxyz, centers, k)
        assert_knn_equal(idx, d2, cnt, i2, d22, c2, sxyz, centers, f"k={k}")
    return oc, sxyz


def test_reference_octree_cloud(port):
    pts = [[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0], [10, 10, 10], [10.1, 10, 10], [10, 10.1, 10], [5, 5, 5], [5, 5, 5.1]]
    oc, sxyz = full_check(port, pts, centers=[[9.9, 9.9, 9.9], [5, 5, 5]])
    idx, d2, cnt = oc.knn(np.array([[9.9, 9.9, 9.9]]), 2)
    assert abs(d2[0, 0] - 0.03) < 1e-4 and sxyz[idx[0, 0], 0] > 9.0          # test_octree.cpp:42-61
    offs, ids = oc.neighborsPrune(np.array([[5.0, 5.0, 5.0]]), 0.25, "square")
    assert len(ids) == 2                                                       # test_octree.cpp:63-80


def test_empty_cloud(port):
    oc, _ = full_check(port, np.zeros((0, 3)), centers=[[0.0, 0.0, 0.0]])
    offs, ids = oc.neighborsPrune(np.zeros((1, 3)), 1.0)
    assert len(ids) == 0
    idx, d2, cnt = oc.knn(np.zeros((1, 3)), 1)
    assert cnt[0] == 0 and idx[0, 0] == 0xFFFFFFFF and np.isinf(d2[0, 0])


@pytest.mark.parametrize("pts", [
    [[1, 1, 1], [1, 1, 1], [2, 2, 2]],                       # duplicates (test_octree_advanced.cpp:49-67)
    [[0, 0, 0], [0, 0, 0], [1, 1, 1]],                       # zero radius (70-83)
    [[0, 0, 0], [10, 10, 10], [5, 5, 5]],                    # boundary (86-101)
    [[1, 1, 1], [2, 0, 0]],                                  # sphere (103-117)
    [[1, 1, 1], [2, 2, 2]],                                  # cube (119-131)
    [[3.5, -2.0, 7.25]],                                     # one point: every axis flat
    [[2.0, 2.0, 2.0]] * 300,                                 # all equal: every sort digit constant
])
def test_reference_advanced_clouds(port, pts):
    full_check(port, pts, leaf=2, centers=np.concatenate([np.asarray(pts, float)[:3], [[0, 0, 0], [10.1, 10.1, 10.1]]]),
               radii=(0.0, 0.01, 1.5, 2.5))


def test_degenerate_line_plane_and_offsets(port):
    line = np.stack([np.arange(100) * 0.1, np.zeros(100), np.zeros(100)], 1)  # test_complex.cpp:37-56
    oc, sxyz = full_check(port, line, leaf=4, centers=[[5.0, 0, 0]], radii=(0.55,))
    assert len(oc.neighborsPrune(np.array([[5.0, 0, 0]]), 0.55, "sphere")[1]) == int(
        np.sum(sq_dist(sxyz, [5.0, 0, 0]) <= 0.55 ** 2))
    g = np.stack(np.meshgrid(np.arange(10) * 0.1, np.arange(10) * 0.1, indexing="ij"), -1).reshape(-1, 2)
    plane = np.concatenate([g, np.zeros((100, 1))], 1)                          # 58-77
    full_check(port, plane, leaf=3, centers=[[0.5, 0.5, 0.0]], radii=(0.2,))
    o = 1e6                                                                     # 79-94
    oc, _ = full_check(port, [[o, o, o], [o + 0.1, o, o], [o, o + 0.1, o]], centers=[[o + 0.05, o + 0.05, o]],
                       radii=(0.1,))
    assert len(oc.neighborsPrune(np.array([[o + 0.05, o + 0.05, o]]), 0.1, "sphere")[1]) == 3


@pytest.mark.parametrize("enc", [1, 5])
def test_points_on_cell_boundaries(port, enc):
    # box [0, 1024]^3: anchor coordinates x * 2048 land exactly on integers (the
    # encoder's exact-division path) and a few ulps either side of them
    rng = np.random.default_rng(11 + enc)
    base = rng.integers(0, 1025, (3000, 3)).astype(np.float64)
    base[0] = 0.0
    base[1] = 1024.0
    nudged = base[2:1500] + rng.choice([-1, 1], (1498, 3)) * np.spacing(base[2:1500]) * rng.integers(1, 4, (1498, 3))
    pts = np.concatenate([base, np.clip(nudged, 0.0, 1024.0)])
    full_check(port, pts, enc=enc, leaf=8, radii=(0.0, 1.0, 7.5), ks=(1, 9))


@pytest.mark.parametrize("enc", [1, 5])
def test_leaf_size_one_and_clusters(port, enc):
    rng = np.random.default_rng(enc)
    pts = np.concatenate([rng.normal(0, 1e-9, (200, 3)), rng.uniform(-5, 5, (300, 3)), np.zeros((50, 3))])
    full_check(port, pts, enc=enc, leaf=1, radii=(0.0, 1e-9, 0.5, 3.0), ks=(1, 7, 60))


def test_device_buffers_match_host_buffers(port):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 50, (20000, 3))
    host = LinearOctree(pts, encoder="hilbert", max_points_leaf=32)
    dev_pts = torch.from_numpy(pts).cuda()
    dev = LinearOctree(dev_pts, encoder="hilbert", max_points_leaf=32)
    assert same_f64(host.box, dev.box)
    L = capi.lib()
    q = torch.from_numpy(pts[:500]).cuda()
    nq = 500
    offs = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")
    total = C.c_uint64()
    st = L.oct_radius_search(dev.handle, 1, 2, q.data_ptr(), nq, None, 2.0, offs.data_ptr(), None, 0,
                             C.byref(total), capi.OCT_MEM_DEVICE)
    assert st == capi.OCT_ERR_CAPACITY
    out = torch.zeros(total.value, dtype=torch.int32, device="cuda")
    st = L.oct_radius_search(dev.handle, 1, 2, q.data_ptr(), nq, None, 2.0, offs.data_ptr(), out.data_ptr(),
                             total.value, C.byref(total), capi.OCT_MEM_DEVICE)
    assert st == capi.OCT_OK and L.oct_synchronize(dev.handle) == capi.OCT_OK
    ho, hi = host.neighborsPrune(pts[:500], 2.0, "sphere")
    assert_csr_equal(offs.cpu().numpy(), out.cpu().numpy().view(np.uint32), ho, hi, "device buffers")
    k = 16
    idx = torch.zeros((nq, k), dtype=torch.int32, device="cuda")
    d2 = torch.zeros((nq, k), dtype=torch.float64, device="cuda")
    cnt = torch.zeros(nq, dtype=torch.int32, device="cuda")
    assert L.oct_knn(dev.handle, q.data_ptr(), nq, k, idx.data_ptr(), d2.data_ptr(), cnt.data_ptr(),
                     capi.OCT_MEM_DEVICE) == capi.OCT_OK
    assert L.oct_synchronize(dev.handle) == capi.OCT_OK
    hi, hd, hc = host.knn(pts[:500], k)
    assert np.array_equal(idx.cpu().numpy().view(np.uint32), hi) and same_f64(d2.cpu().numpy(), hd)


def test_error_statuses(port):
    L = capi.lib()
    p = capi.OctParams(16, 1, 0, 0)
    h = C.c_void_p()
    assert L.oct_cloud_create(C.byref(p), C.byref(h)) == capi.OCT_OK
    # out of order
    assert L.oct_build(h, None) == capi.OCT_ERR_STATE
    assert L.oct_knn(h, None, 0, 1, None, None, None, 0) == capi.OCT_ERR_STATE
    pts = np.random.default_rng(0).uniform(0, 1, (1000, 3))
    assert L.oct_set_points(h, pts.ctypes.data, 1000, 0) == capi.OCT_OK
    assert L.oct_encode_sort(h, None, None, None, None, 0) == capi.OCT_OK
    assert L.oct_build(h, None) == capi.OCT_OK
    q = pts[:4].copy()
    i = np.zeros((4, 2000), np.uint32)
    d = np.zeros((4, 2000))
    assert L.oct_knn(h, q.ctypes.data, 4, 2000, i.ctypes.data, d.ctypes.data, None, 0) == capi.OCT_ERR_INVALID_ARG
    assert L.oct_radius_count(h, 7, 2, q.ctypes.data, 4, None, 1.0, None, 0) == capi.OCT_ERR_INVALID_ARG
    # too small an output buffer: offsets and total still reported
    offs = np.zeros(5, np.uint64)
    out = np.zeros(1, np.uint32)
    tot = C.c_uint64()
    st = L.oct_radius_search(h, 2, 2, q.ctypes.data, 4, None, 0.5, offs.ctypes.data, out.ctypes.data, 1,
                             C.byref(tot), 0)
    assert st == capi.OCT_ERR_CAPACITY and tot.value == offs[-1] and tot.value > 1
    buf = C.create_string_buffer(256)
    assert L.oct_last_error(h, buf, 256) == capi.OCT_OK and b"capacity" in buf.value
    assert L.oct_cloud_destroy(h) == capi.OCT_OK


def test_cloud_pool_trim_between_clouds(port):
    """Clouds reuse the memory destroyed clouds left in the per-device pool; returning it to the
    driver (oct_trim_cloud_memory) between clouds changes no result, and a bad device is refused."""
    from octrees_benchmark_b200.synth import lidar_tile

    L = capi.lib()
    xyz = lidar_tile(40_000, 80.0, 61)
    first = LinearOctree(xyz, encoder="hilbert", max_points_leaf=32)
    want = first.knn(xyz[:300], 8)
    first.close()
    assert L.oct_trim_cloud_memory(0) == capi.OCT_OK
    assert L.oct_trim_cloud_memory(-1) == capi.OCT_ERR_INVALID_ARG
    again = LinearOctree(xyz, encoder="hilbert", max_points_leaf=32)
    got = again.knn(xyz[:300], 8)
    for a, b in zip(want, got):
        assert np.array_equal(a, b)
    again.close()


def test_bounded_device_wait_runs_out_and_reports(port):
    """A device wait on a flag nothing sets gives up after its poll limit and the host reads
    OCT_ERR_DEVICE_LIMIT from the device's error word (no trap, no hang); the device stays usable."""
    from octrees_benchmark_b200.synth import lidar_tile

    L = capi.lib()
    polls = C.c_uint32()
    assert L.oct_device_wait_probe(0, 200_000, C.byref(polls)) == capi.OCT_ERR_DEVICE_LIMIT
    assert polls.value == 200_000
    assert L.oct_device_wait_probe(-1, 10, None) == capi.OCT_ERR_INVALID_ARG
    xyz = lidar_tile(20_000, 60.0, 62)  # the context still runs kernels
    keys, perm, box, sxyz = port.encode_sort(5, xyz)
    oc = LinearOctree(xyz, encoder="hilbert", max_points_leaf=32)
    gk, gp, gx = oc.sorted_points()
    assert np.array_equal(gk, keys)
    oc.close()
