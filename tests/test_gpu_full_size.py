"""Parity at the benchmark's full configurations against the compiled
reference (oracle/_ref: the reference headers built unchanged).

C1: 1,000,000 points (500 m tile, seed 0), Morton, leaf 128; neighborsPrune
    sphere at r = 2.5 and 5.0 m from 10,000 SearchSet centres, full sorted
    sets, on the plain (lanes), packet, packet FP32-filter and batched-engine
    paths.
C2: 10,000,000 points (1.5 km tile, seed 1), Hilbert, leaf 64; every build
    array bitwise; all four kernels x neighbors / neighborsPrune /
    neighborsStruct x r = 1, 2.5, 5 m on 10,000 centres with full sets; the
    radius search over every point of the cloud in order (the reference's
    "-s all") as per-query counts and order-independent set hashes (sphere
    r = 2.5 m, and all four kernels at r = 1 m); kNN k = 10, 50, 250 from
    100,000 centres (squared distances bitwise, ties at the k-th distance by
    lowest index).

The reference runs on every host thread.  Differences are counted per query
(tests/parity.py) and must be zero.
"""
import ctypes as C

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.engine import BatchEngine, Request
from octrees_benchmark_b200.synth import config_cloud, search_set
from tests.parity import csr_count_hash_torch, csr_set_diffs, knn_diffs, ranges_diffs, same_f64

pytestmark = pytest.mark.gpu

KERNELS = {"circle": 0, "sphere": 1, "square": 2, "cube": 3}
ALGOS = {"neighbors": 1, "neighborsPrune": 2, "neighborsStruct": 3}
# (packet, fp32_filter, lanes, kNN in groups)
PATHS = {"lanes8": (False, False, 8, False), "packet": (True, False, 8, True), "packet_fp32": (True, True, 8, True)}


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


@pytest.fixture(scope="module")
def orc():
    from oracle import oracle

    if not oracle.reference_available():
        pytest.skip("oracle/_ref/libref_octree.so is not built (make -C oracle ref REFERENCE=...)")
    return oracle


def set_path(oc, path):
    packet, fp32, lanes, group = PATHS[path]
    oc.set_search_config(packet=packet, fp32_filter=fp32, radius_lanes=lanes, knn_packet=group)


def check_build(oc, R):
    """keys, ids, Box, sorted points and every tree array, bitwise"""
    rx, rids, rkeys = R.points()
    gk, gp, gx = oc.sorted_points()
    assert same_f64(oc.box, R.box())
    assert np.array_equal(gk, rkeys)
    assert np.array_equal(gp.astype(np.uint64), rids)
    assert same_f64(gx, rx)
    assert [oc.n, oc.n_leaf, oc.n_internal, oc.n_total, oc.max_depth_seen] == \
        [R.n, R.n_leaf, R.n_internal, R.n_total, R.max_depth]
    ex, ra = oc.export(), R.arrays()
    assert np.array_equal(ex["offsets"], ra["offsets"])
    assert np.array_equal(ex["ranges"], ra["ranges"])
    for k in ("centers", "radii", "half"):
        assert same_f64(ex[k], ra[k]), k
    return rx


def device_radius(torch, oc, centers_d, kernel, algo, radius):
    """CSR result of a device-resident centre set (OCT_MEM_DEVICE), device tensors."""
    L, h = capi.lib(), oc.handle
    nq = int(centers_d.shape[0])
    offs = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")
    tot = C.c_uint64()
    st = L.oct_radius_search(h, kernel, algo, centers_d.data_ptr(), nq, None, float(radius), offs.data_ptr(), None, 0,
                             C.byref(tot), capi.OCT_MEM_DEVICE)
    assert st in (capi.OCT_OK, capi.OCT_ERR_CAPACITY)
    idx = torch.empty(max(1, tot.value), dtype=torch.int32, device="cuda")
    capi.check(L.oct_radius_search(h, kernel, algo, centers_d.data_ptr(), nq, None, float(radius), offs.data_ptr(),
                                   idx.data_ptr(), tot.value, C.byref(tot), capi.OCT_MEM_DEVICE), h, "radius")
    capi.check(L.oct_synchronize(h), h)
    return offs, idx


# ------------------------------------------------------------------------ C1 --
@pytest.fixture(scope="module")
def c1(torch, orc):
    xyz, cfg = config_cloud("c1_1M_morton")
    R = orc.Reference(cfg["encoder"], xyz, cfg["max_leaf"])
    oc = LinearOctree(xyz, encoder=cfg["encoder"], max_points_leaf=cfg["max_leaf"])
    sxyz = check_build(oc, R)
    q = sxyz[search_set(10_000, len(sxyz))]
    yield oc, R, sxyz, q
    oc.close()


@pytest.mark.parametrize("path", list(PATHS) + ["engine", "engine_fp32"])
def test_c1_prune_sphere_full_sets(torch, c1, path):
    oc, R, sxyz, q = c1
    qd = torch.from_numpy(q).cuda()
    for r in (2.5, 5.0):
        ro, ri = R.radius(1, 2, q, r)
        if path.startswith("engine"):
            set_path(oc, "packet")
            eng = BatchEngine()
            eng.set_config(fp32_filter=path.endswith("fp32"))
            places = eng.run([Request(oc, "radius", qd, radius=r, kernel="sphere", algo="neighborsPrune")])
            offs, idx = eng.radius_result(places[0])
            eng.close()
        else:
            set_path(oc, path)
            offs, idx = oc.radius_search(q, r, "sphere", "neighborsPrune")
        assert csr_set_diffs(offs, idx, ro, ri) == 0, f"{path} r={r}"
        assert int(offs[-1]) == int(ro[-1]) > 0


# ------------------------------------------------------------------------ C2 --
@pytest.fixture(scope="module")
def c2(torch, orc):
    xyz, cfg = config_cloud("c2_10M_hilbert")
    R = orc.Reference(cfg["encoder"], xyz, cfg["max_leaf"])
    oc = LinearOctree(xyz, encoder=cfg["encoder"], max_points_leaf=cfg["max_leaf"])
    del xyz
    sxyz = check_build(oc, R)
    yield oc, R, sxyz
    oc.close()


def test_c2_build_arrays_bitwise(c2):
    oc, R, sxyz = c2  # the fixture checked keys, ids, Box, sorted points and the tree arrays
    assert oc.n == 10_000_000 and oc.n_total > 700_000


@pytest.mark.parametrize("radius", [1.0, 2.5, 5.0])
def test_c2_all_kernels_variants_full_sets(c2, radius):
    oc, R, sxyz = c2
    q = sxyz[search_set(10_000, len(sxyz))]
    for kn, kv in KERNELS.items():
        for algo in ("neighbors", "neighborsPrune"):
            ro, ri = R.radius(kv, ALGOS[algo], q, radius)
            for path in PATHS:
                set_path(oc, path)
                offs, idx = oc.radius_search(q, radius, kn, algo)
                assert csr_set_diffs(offs, idx, ro, ri) == 0, f"{path} {kn} {algo} r={radius}"
        rs_o, rs_p = R.struct_ranges(kv, q, radius)
        for path in PATHS:
            set_path(oc, path)
            go, gp, npts = oc.neighborsStruct(q, radius, kn)
            assert ranges_diffs(go, gp, rs_o, rs_p) == 0, f"{path} {kn} neighborsStruct r={radius}"


@pytest.mark.parametrize("kernel,radius", [("sphere", 2.5), ("sphere", 1.0), ("circle", 1.0), ("square", 1.0),
                                           ("cube", 1.0)])
def test_c2_every_point_count_and_hash(torch, c2, kernel, radius):
    """neighborsPrune with every point of the sorted cloud as a centre, in order, through the
    count-and-hash mode (oct_radius_hash); the first million also as lists, hashed here."""
    oc, R, sxyz = c2
    set_path(oc, "packet")
    kv = KERNELS[kernel]
    rc, rh = R.radius_hash(kv, 2, sxyz, radius)
    chunk = 1 << 20
    bad = 0
    for s in range(0, len(sxyz), chunk):
        qd = torch.from_numpy(np.ascontiguousarray(sxyz[s:s + chunk])).cuda()
        if s == 0:  # the lists, counted and hashed here, on the first chunk
            offs, idx = device_radius(torch, oc, qd, kv, 2, radius)
            lc, lh = csr_count_hash_torch(offs, idx)
            del offs, idx
        gc, gh = oc.radius_hash(qd, radius, kernel, "neighborsPrune")  # counts and hashes on the device
        if s == 0:
            assert torch.equal(gc, lc.to(gc.dtype)) and torch.equal(gh, lh.to(gh.dtype))
        gc = gc.cpu().numpy().view(np.uint64)
        gh = gh.cpu().numpy().view(np.uint64)
        m = len(gc)
        bad += int(((gc != rc[s:s + m]) | (gh != rh[s:s + m])).sum())
    assert bad == 0, f"{bad} of {len(sxyz)} queries differ"
    assert rc.sum() > len(sxyz)


@pytest.mark.parametrize("k", [10, 50, 250])
def test_c2_knn_from_100k_centres(torch, c2, k):
    oc, R, sxyz = c2
    q = sxyz[search_set(100_000, len(sxyz))]
    ki, kd, kc = R.knn(q, k)
    for path in list(PATHS) + ["engine"]:
        if path == "engine":
            set_path(oc, "packet")
            eng = BatchEngine()
            places = eng.run([Request(oc, "knn", torch.from_numpy(q).cuda(), k=k)])
            idx, d2, cnt = eng.knn_result(places[0], k)
            eng.close()
        else:
            set_path(oc, path)
            idx, d2, cnt = oc.knn(q, k)
        diffs, err, _ = knn_diffs(idx, d2, cnt, ki, kd, kc, sxyz, q)
        assert diffs == 0 and err == 0.0, f"{path} k={k}: {diffs} queries differ, max d2 error {err}"
