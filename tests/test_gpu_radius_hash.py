"""oct_radius_hash: per-centre neighbour counts and order-independent set
hashes (sum of splitmix64's output function over the neighbour indices,
mod 2^64) without the neighbour lists, against the compiled reference
(the bridge's refo_radius_hash runs the reference's own neighbors /
neighborsPrune and hashes what it returns), for the four kernels, host and
device buffers, and against the lists oct_radius_search returns."""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.synth import lidar_tile
from tests.parity import mix64_np

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(1, 32), (5, 64)], ids=["morton32", "hilbert64"])
def clouds(request):
    from oracle import oracle

    if not oracle.reference_available():
        pytest.skip("oracle/_ref is not built")
    enc, leaf = request.param
    xyz = lidar_tile(200_000, 150.0, seed=17)
    R = oracle.Reference(enc, xyz, leaf)
    oc = LinearOctree(xyz, encoder=enc, max_points_leaf=leaf)
    yield oc, R
    oc.close()


@pytest.mark.parametrize("kernel", ["sphere", "circle", "cube", "square"])
def test_hash_matches_reference(clouds, kernel):
    oc, R = clouds
    sxyz = R.points()[0]
    rng = np.random.default_rng(3)
    q = np.concatenate([sxyz[rng.integers(0, len(sxyz), 4000)], rng.uniform(sxyz.min(0) - 5, sxyz.max(0) + 5,
                                                                             (500, 3))])
    kv = capi.KERNELS[kernel]
    for algo in ("neighbors", "neighborsPrune"):
        for radius in (0.0, 1.0, 4.0):
            rc, rh = R.radius_hash(kv, capi.ALGOS[algo], q, radius)
            gc, gh = oc.radius_hash(q, radius, kernel, algo)
            assert np.array_equal(gc, rc), f"{kernel} {algo} r={radius} counts"
            assert np.array_equal(gh, rh), f"{kernel} {algo} r={radius} hashes"
    assert rc.sum() > len(q)


def test_hash_equals_lists_and_device_buffers(clouds):
    torch = pytest.importorskip("torch")
    oc, R = clouds
    sxyz = R.points()[0]
    q = sxyz[::37]
    offs, idx = oc.radius_search(q, 2.5, "sphere", "neighborsPrune")
    want_c = np.diff(offs).astype(np.uint64)
    csum = np.concatenate([np.zeros(1, np.uint64), np.cumsum(mix64_np(idx.astype(np.uint64)), dtype=np.uint64)])
    want_h = csum[offs[1:].astype(np.int64)] - csum[offs[:-1].astype(np.int64)]  # wraps mod 2^64, as the hash
    gc, gh = oc.radius_hash(q, 2.5, "sphere", "neighborsPrune")
    assert np.array_equal(gc, want_c) and np.array_equal(gh, want_h)
    sc, sh = oc.radius_hash(q, 2.5, "sphere", "neighborsStruct")  # the expanded ranges: the same set
    assert np.array_equal(sc, want_c) and np.array_equal(sh, want_h)
    dc, dh = oc.radius_hash(torch.from_numpy(np.ascontiguousarray(q)).cuda(), 2.5, "sphere", "neighborsPrune")
    assert np.array_equal(dc.cpu().numpy().view(np.uint64), want_c)
    assert np.array_equal(dh.cpu().numpy().view(np.uint64), want_h)
    e0c, e0h = oc.radius_hash(np.zeros((0, 3)), 2.5, "sphere", "neighborsPrune")
    assert len(e0c) == 0 and len(e0h) == 0


def test_engine_hash_copy_out(clouds):
    """oct_engine_copy_radius_hash: the counts and hashes of a batched radius request equal the
    single-cloud oct_radius_hash ones (and thus the reference's)."""
    torch = pytest.importorskip("torch")
    from octrees_benchmark_b200.engine import BatchEngine, Request

    oc, R = clouds
    sxyz = R.points()[0]
    q = np.ascontiguousarray(sxyz[::29])
    dq = torch.from_numpy(q).cuda()
    eng = BatchEngine()
    try:
        places = eng.run([Request(oc, "radius", dq, radius=3.0, kernel="cube", algo="neighbors"),
                          Request(oc, "knn", dq, k=8),
                          Request(oc, "radius", dq[:1000].contiguous(), radius=1.5, kernel="sphere")])
        for pl, (r, kern, algo, n) in zip((places[0], places[2]), ((3.0, "cube", "neighbors", len(q)),
                                                                 (1.5, "sphere", "neighborsPrune", 1000))):
            gc, gh = eng.radius_hash_result(pl)
            wc, wh = oc.radius_hash(q[:n], r, kern, algo)
            assert np.array_equal(gc, wc) and np.array_equal(gh, wh)
        with pytest.raises(capi.OctError):
            eng.radius_hash_result(places[1])  # a kNN request's place
    finally:
        eng.close()
