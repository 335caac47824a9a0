"""The batched multi-cloud engine (oct_engine_*) through the C ABI.

A batch mixes clouds (Morton and Hilbert keys, several leaf sizes), radius
requests of every kernel with neighbors and neighborsPrune (one radius or one
per centre), kNN requests with k on both sides of the 32 and 64 boundaries (the
register lists and the shared-memory lists), and empty requests.  Every request's result must be bitwise the single-cloud call's
result (neighbour lists in the same ascending order, kNN indices and squared
distances identical), and two of them are also checked against the oracle.
The same batch through the captured graph, its replay, the direct launch
sequence, the FP32 filter, a result array that has to grow, and the
autotuner's configuration all give the same bits.
"""
import ctypes as C

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.engine import BatchEngine, Request
from octrees_benchmark_b200.synth import lidar_tile, query_indices
from tests.parity import assert_csr_equal, assert_knn_equal

pytestmark = pytest.mark.gpu

KERNELS = ["circle", "sphere", "square", "cube"]


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


@pytest.fixture(scope="module")
def clouds():
    specs = [(3_001, 25.0, 11, "morton", 16), (20_000, 60.0, 12, "hilbert", 32), (45_000, 80.0, 13, "hilbert", 64),
             (9_000, 40.0, 14, "morton", 128), (60_000, 90.0, 15, "morton", 32)]
    out = []
    for n, tile, seed, enc, leaf in specs:
        oc = LinearOctree(lidar_tile(n, tile, seed), encoder=enc, max_points_leaf=leaf)
        _, _, sxyz = oc.sorted_points()
        out.append((oc, sxyz))
    return out


def centres(torch, sxyz, nq, seed):
    c = sxyz[query_indices(nq, len(sxyz), seed)]
    return c, torch.from_numpy(np.ascontiguousarray(c)).cuda()


def mixed_batch(torch, clouds, seed=0):
    """Requests over every cloud: radius with each kernel/algo, kNN k in {1, 10, 33, 64, 65, 250}, empties."""
    rng = np.random.default_rng(seed)
    reqs, host = [], []
    for ci, (oc, sxyz) in enumerate(clouds):
        for j, kern in enumerate(KERNELS):
            nq = int(rng.integers(1, 400))
            c, dc = centres(torch, sxyz, nq, 100 * ci + j)
            algo = "neighborsPrune" if (ci + j) % 2 == 0 else "neighbors"
            if j % 2:
                r = rng.uniform(0.5, 3.0, nq)
                reqs.append(Request(oc, "radius", dc, radii=torch.from_numpy(r).cuda(), kernel=kern, algo=algo))
                host.append(("radius", ci, c, r, kern, algo))
            else:
                r = float(rng.uniform(0.5, 3.0))
                reqs.append(Request(oc, "radius", dc, radius=r, kernel=kern, algo=algo))
                host.append(("radius", ci, c, r, kern, algo))
        for k in (1, 10, 33, 64, 65, 250):
            nq = int(rng.integers(1, 300))
            c, dc = centres(torch, sxyz, nq, 1000 + 10 * ci + k)
            reqs.append(Request(oc, "knn", dc, k=k))
            host.append(("knn", ci, c, k))
    # empty requests of both kinds
    empty = torch.zeros((0, 3), dtype=torch.float64, device="cuda")
    reqs.insert(3, Request(clouds[0][0], "radius", empty, radius=1.0))
    host.insert(3, ("radius", 0, np.zeros((0, 3)), 1.0, "sphere", "neighborsPrune"))
    reqs.append(Request(clouds[1][0], "knn", empty, k=5))
    host.append(("knn", 1, np.zeros((0, 3)), 5))
    return reqs, host


def single_cloud(clouds, h):
    oc = clouds[h[1]][0]
    if h[0] == "radius":
        _, _, c, r, kern, algo = h
        return oc.radius_search(c, r, kern, algo)
    _, _, c, k = h
    return oc.knn(c, k)


def engine_results(eng, places, host):
    out = []
    for pl, h in zip(places, host):
        out.append(eng.radius_result(pl) if h[0] == "radius" else eng.knn_result(pl, h[3]))
    return out


def assert_same(a, b, what):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.dtype == y.dtype and np.array_equal(x, y), what


def test_engine_matches_single_cloud_calls(torch, clouds):
    reqs, host = mixed_batch(torch, clouds)
    eng = BatchEngine()
    places = eng.run(reqs)
    got = engine_results(eng, places, host)
    for i, h in enumerate(host):
        want = single_cloud(clouds, h)
        if h[0] == "radius":
            assert np.array_equal(got[i][0], want[0]), f"request {i}: offsets"
            assert np.array_equal(got[i][1], want[1]), f"request {i}: indices"
            assert places[i].n_results == len(want[1])
        else:
            assert_same(got[i], want, f"request {i}: kNN")
    assert eng.radius_total == sum(pl.n_results for pl, h in zip(places, host) if h[0] == "radius")


def test_engine_matches_oracle(torch, clouds, port):
    oc, sxyz = clouds[2]
    c, dc = centres(torch, sxyz, 500, 7)
    eng = BatchEngine()
    pl = eng.run([Request(oc, "radius", dc, radius=2.0, kernel="sphere", algo="neighborsPrune"),
                  Request(oc, "knn", dc, k=50)])
    keys, _, _ = oc.sorted_points()
    tree = port.build(5, keys, oc.max_points_leaf, oc.box)
    ro, ri = tree.radius(sxyz, 1, 2, c, 2.0)
    go, gi = eng.radius_result(pl[0])
    assert_csr_equal(go, gi, ro, ri, "engine radius vs oracle")
    idx, d2, cnt = eng.knn_result(pl[1], 50)
    oi, od, ocnt = tree.knn(sxyz, c, 50)
    assert_knn_equal(idx, d2, cnt, oi, od, ocnt, sxyz, c, "engine kNN vs oracle")


@pytest.mark.parametrize("one_cloud", [False, True])
def test_group_knn_matches_per_query(torch, clouds, one_cloud):
    """kNN in groups of queries per warp (runs of seeded groups, requests that end mid-group,
    the fallback group for centres whose provisional threshold undershoots) against one warp
    per query, on a multi-cloud batch and on a one-cloud batch."""
    rng = np.random.default_rng(5)
    use = [2] if one_cloud else range(len(clouds))
    reqs, host = [], []
    for ci in use:
        oc, sxyz = clouds[ci]
        for k in (1, 10, 32, 33, 50, 64):
            nq = int(rng.integers(1, 3000))
            c, _ = centres(torch, sxyz, nq, 2000 + 10 * ci + k)
            c = c.copy()
            c[::17, 2] += 40.0  # above the terrain: fewer than k points near the first cells
            reqs.append(Request(oc, "knn", torch.from_numpy(c).cuda(), k=k))
            host.append(("knn", ci, c, k))
    eng_g, eng_q = BatchEngine(), BatchEngine()
    eng_g.set_config(knn_group=True, knn_bucket=256)
    eng_q.set_config(knn_group=False, knn_bucket=256)
    got_g = engine_results(eng_g, eng_g.run(reqs), host)
    got_q = engine_results(eng_q, eng_q.run(reqs), host)
    for i, (a, b) in enumerate(zip(got_g, got_q)):
        assert_same(a, b, f"group vs per-query, request {i}")
    for i in range(0, len(host), 5):
        assert_same(got_g[i], single_cloud(clouds, host[i]), f"group vs single-cloud call, request {i}")


def test_graph_replay_direct_and_fp32_agree(torch, clouds):
    reqs, host = mixed_batch(torch, clouds, seed=1)
    eng = BatchEngine()
    base = engine_results(eng, eng.run(reqs), host)
    replay = engine_results(eng, eng.run(reqs), host)  # the captured graph, replayed
    direct_eng = BatchEngine(graph=False)
    direct = engine_results(direct_eng, direct_eng.run(reqs), host)
    eng.set_config(fp32_filter=True, knn_bucket=0, radius_blocks_per_sm=4, knn_blocks_per_sm=8)
    fp32 = engine_results(eng, eng.run(reqs), host)
    runs = [(replay, "replay"), (direct, "direct"), (fp32, "fp32/bucket0")]
    for sel in (capi.OCT_FP32_RADIUS, capi.OCT_FP32_KNN):  # one filter at a time
        eng.set_config(fp32_filter=sel, knn_bucket=256)
        assert eng.config()["fp32_filter"] == sel
        runs.append((engine_results(eng, eng.run(reqs), host), f"fp32 selector {sel}"))
    for other, name in runs:
        for i, (a, b) in enumerate(zip(base, other)):
            assert_same(a, b, f"{name}, request {i}")


def test_result_array_grows_and_batch_reruns(torch, clouds):
    oc, sxyz = clouds[4]
    c, dc = centres(torch, sxyz, 2000, 9)
    eng = BatchEngine(reserve_results=1000)  # far below the ~10^5 results
    pl = eng.run([Request(oc, "radius", dc, radius=3.0, kernel="cube")])
    assert pl[0].n_results > 1000
    got = eng.radius_result(pl[0])
    want = oc.radius_search(c, 3.0, "cube", "neighborsPrune")
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_many_requests_use_the_request_digits(torch, clouds):
    """300 requests: the sort keys carry a second request byte."""
    reqs, host = [], []
    for i in range(300):
        oc, sxyz = clouds[i % len(clouds)]
        c, dc = centres(torch, sxyz, 1 + (i * 7) % 50, 5000 + i)
        if i % 3:
            reqs.append(Request(oc, "radius", dc, radius=1.5, kernel=KERNELS[i % 4]))
            host.append(("radius", i % len(clouds), c, 1.5, KERNELS[i % 4], "neighborsPrune"))
        else:
            reqs.append(Request(oc, "knn", dc, k=12))
            host.append(("knn", i % len(clouds), c, 12))
    eng = BatchEngine()
    got = engine_results(eng, eng.run(reqs), host)
    for i, h in enumerate(host):
        want = single_cloud(clouds, h)
        assert_same(got[i], want, f"request {i}")


def test_autotune_keeps_results(torch, clouds):
    reqs, host = mixed_batch(torch, clouds, seed=2)
    eng = BatchEngine()
    base = engine_results(eng, eng.run(reqs), host)
    cfg = eng.autotune(reqs)
    assert cfg["radius_blocks_per_sm"] in (4, 8, 12) and cfg["knn_bucket"] in (0, 64, 128, 256)
    tuned = engine_results(eng, eng.run(reqs), host)
    for i, (a, b) in enumerate(zip(base, tuned)):
        assert_same(a, b, f"autotuned, request {i}")
    assert eng.last_ms > 0


def test_engine_rejects_bad_requests(torch, clouds):
    oc, sxyz = clouds[0]
    _, dc = centres(torch, sxyz, 10, 3)
    eng = BatchEngine()
    for bad in (Request(oc, "knn", dc, k=0), Request(oc, "knn", dc, k=1025),
                Request(oc, "radius", dc, radius=1.0, algo="neighborsStruct")):
        with pytest.raises(capi.OctError) as ei:
            eng.run([bad])
        assert ei.value.status == capi.OCT_ERR_INVALID_ARG
    # a cloud that has points but no tree
    L = capi.lib()
    h = C.c_void_p()
    capi.check(L.oct_cloud_create(C.byref(capi.OctParams(32, 1, 0, 0)), C.byref(h)))
    try:
        r = capi.OctRequest()
        r.cloud = h.value
        r.type = capi.OCT_REQ_KNN
        r.k = 3
        r.centers = dc.data_ptr()
        r.nq = 10
        st = L.oct_engine_run(eng._h, C.byref(r), 1, None, None)
        assert st == capi.OCT_ERR_STATE
    finally:
        L.oct_cloud_destroy(h)
    # the engine still works after the rejections
    pl = eng.run([Request(oc, "knn", dc, k=3)])
    assert pl[0].nq == 10
