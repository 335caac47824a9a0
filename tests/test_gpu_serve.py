"""The serving scheduler (oct_server_*) through the C ABI.

Requests submitted together are batched continuously, several batches in
flight on different streams; every request's result must be bitwise the
result of the same request run alone (the single-cloud call), in the batched
server and in the plain one-request-per-launch server.  A tight HBM budget
makes requests wait (admission stalls) without changing any result; owned
clouds are evicted least recently used first when a new cloud does not fit;
removing a cloud waits for its running requests.
"""
import ctypes as C

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.engine import Request
from octrees_benchmark_b200.serve import Server
from octrees_benchmark_b200.synth import lidar_tile, query_indices

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


@pytest.fixture(scope="module")
def clouds(torch):
    specs = [(30_000, 70.0, 21, "hilbert", 32), (80_000, 120.0, 22, "morton", 64), (12_000, 40.0, 23, "hilbert", 16),
             (50_000, 90.0, 24, "morton", 128)]
    out = []
    for n, tile, seed, enc, leaf in specs:
        oc = LinearOctree(lidar_tile(n, tile, seed), encoder=enc, max_points_leaf=leaf)
        _, _, sxyz = oc.sorted_points()
        out.append((oc, sxyz))
    return out


def make_requests(torch, clouds, n=60, seed=3):
    rng = np.random.default_rng(seed)
    reqs, host = [], []
    for i in range(n):
        ci = int(rng.integers(0, len(clouds)))
        oc, sxyz = clouds[ci]
        nq = int(np.exp(rng.uniform(0, np.log(3000))))
        c = sxyz[query_indices(nq, len(sxyz), 100 + i)]
        dc = torch.from_numpy(np.ascontiguousarray(c)).cuda()
        if rng.random() < 0.5:
            r = float(rng.uniform(0.5, 4.0))
            kern = ["sphere", "cube", "circle", "square"][i % 4]
            reqs.append(Request(oc, "radius", dc, radius=r, kernel=kern, algo="neighborsPrune"))
            host.append(("radius", ci, c, r, kern))
        else:
            k = int(rng.choice([10, 50, 250]))
            reqs.append(Request(oc, "knn", dc, k=k))
            host.append(("knn", ci, c, k))
    return reqs, host


def alone(clouds, h):
    oc = clouds[h[1]][0]
    if h[0] == "radius":
        return oc.radius_search(h[2], h[3], h[4], "neighborsPrune")
    return oc.knn(h[2], h[3])


def serve_all(srv, reqs, host):
    """Submit everything at once, collect every completion, copy results, release."""
    tickets = [srv.submit(r) for r in reqs]
    by_ticket = {t: i for i, t in enumerate(tickets)}
    results = [None] * len(reqs)
    got = 0
    for _ in range(2000):
        for c in srv.poll(256, wait_ms=20):
            i = by_ticket[c["ticket"]]
            assert c["status"] == capi.OCT_OK, c
            h = host[i]
            if h[0] == "radius":
                results[i] = srv.radius_result(c["ticket"], c["nq"], c["n_results"])
            else:
                results[i] = srv.knn_result(c["ticket"], c["nq"], h[3])
            assert c["latency_ms"] >= c["queue_ms"] >= 0.0
            srv.release(c["ticket"])
            got += 1
        if got == len(reqs):
            break
    assert got == len(reqs)
    return results


def check_same(results, clouds, host):
    for i, h in enumerate(host):
        want = alone(clouds, h)
        for a, b in zip(results[i], want):
            assert a.dtype == b.dtype and np.array_equal(a, b), f"request {i} ({h[0]}) differs from its solo run"


@pytest.mark.parametrize("plain", [False, True], ids=["batched", "plain"])
def test_results_same_alone_and_in_the_mix(torch, clouds, plain):
    reqs, host = make_requests(torch, clouds)
    srv = Server(plain=plain, slots=3, max_batch_requests=7)
    for oc, _ in clouds:
        srv.add_cloud(oc)
    results = serve_all(srv, reqs, host)
    st = srv.stats()
    srv.close()
    if not plain:
        assert st["batches"] >= len(reqs) // 7
    else:
        assert st["batches"] == len(reqs)
    assert st["completed"] == st["submitted"] == len(reqs)
    # the plain server switched the clouds to the plain path; the solo runs below use it too
    check_same(results, clouds, host)


def test_tight_budget_stalls_admission_without_changing_results(torch, clouds):
    reqs, host = make_requests(torch, clouds, n=30, seed=5)
    cloud_bytes = 0
    for oc, _ in clouds:
        b = C.c_uint64()
        capi.lib().oct_cloud_memory(oc.handle, C.byref(b))
        cloud_bytes += b.value
    srv = Server(slots=3, hbm_budget=cloud_bytes + (2 << 20))  # room for about one small batch at a time
    for oc, _ in clouds:
        srv.add_cloud(oc)
    results = serve_all(srv, reqs, host)
    st = srv.stats()
    srv.close()
    assert st["admission_stalls"] > 0
    assert st["peak_bytes"] <= cloud_bytes + (2 << 20) or st["batches"] > 1
    check_same(results, clouds, host)


def test_owned_clouds_are_evicted_lru_and_removal_waits(torch):
    L = capi.lib()
    made = [LinearOctree(lidar_tile(20_000, 50.0, 40 + i), encoder="hilbert", max_points_leaf=32) for i in range(3)]
    sizes = []
    for oc in made:
        b = C.c_uint64()
        L.oct_cloud_memory(oc.handle, C.byref(b))
        sizes.append(b.value)
    srv = Server(slots=2, hbm_budget=sizes[0] + sizes[1] + sizes[2] // 2)
    handles = [oc.handle.value for oc in made]
    srv.add_cloud(made[0], owned=True)
    srv.add_cloud(made[1], owned=True)
    # a request on cloud 1 makes cloud 0 the least recently used one
    c = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    t = srv.submit(Request(_H(handles[1]), "knn", c, k=3))
    srv.add_cloud(made[2], owned=True)  # does not fit: cloud 0 (idle, oldest) is evicted
    assert srv.stats()["evictions"] == 1
    with pytest.raises(capi.OctError) as ei:
        srv.submit(Request(_H(handles[0]), "knn", c, k=3))
    assert ei.value.status == capi.OCT_ERR_STATE
    for comp in srv.poll(16, wait_ms=2000):
        srv.release(comp["ticket"])
    srv.remove_cloud(C.c_void_p(handles[1]))  # idle now: removed (and destroyed)
    assert srv.stats()["cloud_bytes"] == sizes[2]
    srv.close()


def test_bad_requests_are_rejected(torch, clouds):
    oc, sxyz = clouds[0]
    srv = Server()
    c = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(capi.OctError) as ei:  # not registered
        srv.submit(Request(oc, "knn", c, k=3))
    assert ei.value.status == capi.OCT_ERR_STATE
    srv.add_cloud(oc)
    for bad in (Request(oc, "knn", c, k=0), Request(oc, "knn", c, k=2000),
                Request(oc, "radius", c, radius=1.0, algo="neighborsStruct")):
        with pytest.raises(capi.OctError) as ei:
            srv.submit(bad)
        assert ei.value.status == capi.OCT_ERR_INVALID_ARG
    srv.close()


def test_replay_inserts_clouds_while_batches_capture(torch):
    """Clouds built by a background thread and inserted while the scheduler
    captures and replays batch graphs (a batch on one cloud is captured per
    cloud, so every insert brings new captures): the replay ends by itself,
    every request completes and every insertion lands."""
    from octrees_benchmark_b200.serve import ServingWorkload, replay

    wl = ServingWorkload(seconds=3.0, rate=300.0, n_clouds=3, insert_every=0.5, pool=4000, workers=1,
                         cloud_points=(40_000, 120_000), insert_points=(30_000, 80_000), max_batch=2000)
    epochs = {int(it.t // wl.insert_every) for it in wl.stream} - {0}
    srv = Server(slots=3)
    try:
        res = replay(wl, srv, drain_s=30.0, insert_wait_s=60.0)
    finally:
        srv.close()
    assert res["errors"] == 0 and res["insert_failures"] == 0 and res["skipped"] == 0
    assert res["completed"] == res["requests"] and res["unfinished"] == 0
    assert res["clouds_inserted"] == len(epochs) and len(epochs) >= 4


class _H:
    def __init__(self, h):
        self.handle = C.c_void_p(h)
