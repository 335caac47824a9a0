"""Parity of the CUDA path against the reference's outputs (golden fixtures)
and the CPU oracle, through the C ABI.  Bit-exact: keys, sort permutation, Box,
octree arrays, every neighbour set (as sorted index sets), neighborsStruct
ranges, kNN squared distances (ties at the k-th distance by lowest index)."""
import glob
import os

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.synth import lidar_tile, query_indices
from tests.parity import assert_csr_equal, assert_knn_equal, assert_ranges_equal, same_f64

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CLOUDS = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if not p.endswith("keys_anchor.npz"))
KERNELS = {"sphere": 1, "circle": 0, "cube": 3, "square": 2}
ALGO_NAMES = {1: "neighbors", 2: "neighborsPrune", 3: "neighborsStruct"}
# search paths: (packet, fp32_filter, lanes per query of the non-packet path, kNN in groups, kNN bucket)
PATHS = {"lanes8": (False, False, 8, False, 256), "lanes16": (False, False, 16, False, 256),
         "lanes32": (False, False, 32, False, 256), "packet": (True, False, 8, False, 256),
         "packet_fp32": (True, True, 8, False, 256), "knn_packet": (True, False, 8, True, 256),
         "knn_packet_fp32": (True, True, 8, True, 256),
         # one FP32 filter at a time (2: the radius filter, 3: the kNN filter)
         "packet_fp32_radius": (True, 2, 8, True, 256), "packet_fp32_knn": (True, 3, 8, True, 256),
         "knn_leaves": (True, False, 8, False, 0), "knn_bucket2k": (True, False, 8, False, 2048)}


def octree(xyz, enc, leaf, path):
    packet, fp32, lanes, knn_packet, bucket = PATHS[path]
    return LinearOctree(xyz, encoder=enc, max_points_leaf=leaf, radius_group=lanes, packet=packet, fp32_filter=fp32,
                        knn_packet=knn_packet, knn_bucket=bucket)


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def check_cloud_against(oc, keys, ids, box, sxyz, info, arrays):
    gk, gp, gx = oc.sorted_points()
    assert same_f64(oc.box, box)
    assert np.array_equal(gk, keys)
    assert np.array_equal(gp.astype(np.uint64), np.asarray(ids, np.uint64))
    assert same_f64(gx, sxyz)
    assert [oc.n, oc.n_leaf, oc.n_internal, oc.n_total, oc.max_depth_seen] == [int(v) for v in info]
    ex = oc.export()
    assert np.array_equal(ex["offsets"], arrays["offsets"])
    assert np.array_equal(ex["ranges"], np.asarray(arrays["ranges"], np.uint64))
    for k in ("centers", "radii", "half"):
        assert same_f64(ex[k], arrays[k]), k


@pytest.mark.parametrize("path", CLOUDS, ids=[os.path.basename(p)[:-4] for p in CLOUDS])
@pytest.mark.parametrize("search", ["lanes8", "lanes32", "packet", "packet_fp32"])
def test_gpu_matches_reference_fixture(path, search):
    g = load(path)
    oc = octree(g["xyz"], int(g["encoder"]), int(g["max_leaf"]), search)
    arrays = {k[5:]: v for k, v in g.items() if k.startswith("tree_")}
    check_cloud_against(oc, g["keys"], g["ids"], g["box"], g["sorted_xyz"], g["info"], arrays)
    q = g["centers"]
    sxyz = g["sorted_xyz"]
    for ri, r in enumerate(g["radii"]):
        for kn in KERNELS:
            for algo in (1, 2, 3):
                offs, idx = oc.radius_search(q, r, kn, ALGO_NAMES[algo])
                assert_csr_equal(offs, idx, g[f"rad_{ri}_{kn}_{algo}_offs"], g[f"rad_{ri}_{kn}_{algo}_idx"],
                                 f"{kn} {ALGO_NAMES[algo]} r={r}")
                cnt = oc.radius_count(q, r, kn, ALGO_NAMES[algo])
                assert np.array_equal(cnt, np.diff(g[f"rad_{ri}_{kn}_{algo}_offs"].astype(np.int64)))
            ro, pairs, npts = oc.neighborsStruct(q, r, kn)
            assert_ranges_equal(ro, pairs, g[f"struct_{ri}_{kn}_offs"], g[f"struct_{ri}_{kn}_pairs"], kn)
            assert np.array_equal(npts, np.diff(g[f"rad_{ri}_{kn}_3_offs"].astype(np.int64)))
    for k in g["ks"]:
        k = int(k)
        idx, d2, cnt = oc.knn(q, k)
        assert_knn_equal(idx, d2, cnt, g[f"knn_{k}_idx"], g[f"knn_{k}_d2"], g[f"knn_{k}_cnt"], sxyz, q, f"k={k}")
    oc.close()


SYNTH = [
    # (n, tile, seed, encoder, leaf)
    (200_000, 220.0, 31, 5, 64),
    (200_000, 220.0, 32, 1, 128),
    (50_000, 60.0, 33, 5, 16),
    (30_000, 50.0, 34, 1, 1),
]


@pytest.fixture(scope="module")
def synth_cases(port):
    out = []
    for n, tile, seed, enc, leaf in SYNTH:
        xyz = lidar_tile(n, tile, seed)
        if leaf == 1:
            xyz[::5] = xyz[11]  # exact duplicates force level-21 leaves
        keys, perm, box, sxyz = port.encode_sort(enc, xyz)
        t = port.build(enc, keys, leaf, box)
        out.append((xyz, enc, leaf, keys, perm, box, sxyz, t))
    return out


@pytest.mark.parametrize("case", range(len(SYNTH)))
def test_gpu_build_matches_oracle(synth_cases, case):
    xyz, enc, leaf, keys, perm, box, sxyz, t = synth_cases[case]
    oc = LinearOctree(xyz, encoder=enc, max_points_leaf=leaf)
    info = [t.n, t.n_leaf, t.n_internal, t.n_total, t.max_depth]
    check_cloud_against(oc, keys, perm, box, sxyz, info, t.arrays())
    oc.close()


@pytest.mark.parametrize("enc", [1, 5])
def test_gpu_build_dense_cluster(port, enc):
    """20k of 40k points inside one tiny cell (most with equal keys): the sort
    keeps them in input order and the deep leaves match the oracle."""
    xyz = lidar_tile(40_000, 80.0, 35)
    xyz[:20_000] = xyz[7] + 1e-9 * np.arange(20_000, dtype=np.float64)[:, None]
    keys, perm, box, sxyz = port.encode_sort(enc, xyz)
    t = port.build(enc, keys, 32, box)
    oc = LinearOctree(xyz, encoder=enc, max_points_leaf=32)
    info = [t.n, t.n_leaf, t.n_internal, t.n_total, t.max_depth]
    check_cloud_against(oc, keys, perm, box, sxyz, info, t.arrays())
    oc.close()


@pytest.mark.parametrize("n", [1, 2, 100, 3071, 3072, 3073, 4607, 4608, 4609, 8193, 9217, 70_000])
def test_gpu_sort_sizes(port, n):
    """Keys, order and sorted points at sizes around the sort's 4608-key tiles
    (and the 3072-key tiles of its earlier shape) and its single-tile and
    many-tile cases."""
    xyz = lidar_tile(max(n, 2), 120.0, 36)[:n]
    keys, perm, box, sxyz = port.encode_sort(5, xyz)
    oc = LinearOctree(xyz, encoder="hilbert", max_points_leaf=64)
    gk, gp, gx = oc.sorted_points()
    assert np.array_equal(gk, keys)
    assert np.array_equal(gp.astype(np.uint64), np.asarray(perm, np.uint64))
    assert same_f64(gx, sxyz)
    oc.close()


@pytest.mark.parametrize("case", range(len(SYNTH)))
@pytest.mark.parametrize("search", [p for p in PATHS if not p.startswith("knn")])
def test_gpu_radius_matches_oracle(synth_cases, case, search):
    xyz, enc, leaf, keys, perm, box, sxyz, t = synth_cases[case]
    oc = octree(xyz, enc, leaf, search)
    q = sxyz[query_indices(400, len(sxyz), seed=case)]
    # also centres that are not cloud points, some far outside the cloud
    rng = np.random.default_rng(case)
    q = np.concatenate([q, q[:60] + rng.normal(0, 2.0, (60, 3)), box[6:9] - 3.0 + rng.uniform(0, 1, (4, 3))])
    radii = [0.5, 2.5, 5.0] if search in ("lanes8", "packet", "packet_fp32") else [2.5]
    for r in radii:
        for kn, kv in KERNELS.items():
            for algo in (1, 2, 3):
                offs, idx = oc.radius_search(q, r, kn, ALGO_NAMES[algo])
                o2, i2 = t.radius(sxyz, kv, algo, q, r)
                assert_csr_equal(offs, idx, o2, i2, f"{kn} {ALGO_NAMES[algo]} r={r}")
                # every query's output is ascending (octants are visited in key order)
                d = np.diff(idx.astype(np.int64))
                mask = np.ones(len(d), bool)
                starts = offs[1:-1].astype(np.int64)
                mask[starts[(starts >= 1) & (starts <= len(d))] - 1] = False
                assert np.all(d[mask] > 0)
            ro, pairs, npts = oc.neighborsStruct(q, r, kn)
            o2, p2 = t.struct_ranges(sxyz, kv, q, r)
            assert_ranges_equal(ro, pairs, o2, p2, kn)
    # per-query radii
    rr = np.random.default_rng(case).uniform(0.5, 5.0, len(q))
    for kn, kv in KERNELS.items():
        offs, idx = oc.neighborsPrune(q, rr, kn)
        o2, i2 = t.radius(sxyz, kv, 2, q, rr)
        assert_csr_equal(offs, idx, o2, i2, f"per-query radii {kn}")
    if search == "packet_fp32":
        tests, retests = oc.search_stats()
        assert tests > 0 and retests < tests  # the band catches few points
    oc.close()


@pytest.mark.parametrize("case", range(len(SYNTH)))
@pytest.mark.parametrize("search", ["lanes8", "lanes32", "packet"])
def test_gpu_approx_matches_oracle(synth_cases, case, search):
    """neighborsApprox: the ranges at every cut level, both bounds, every kernel; and the
    lower-bound points within the exact set within the upper-bound points."""
    xyz, enc, leaf, keys, perm, box, sxyz, t = synth_cases[case]
    oc = octree(xyz, enc, leaf, search)
    q = sxyz[query_indices(200, len(sxyz), seed=case)]
    rng = np.random.default_rng(case)
    q = np.concatenate([q, q[:30] + rng.normal(0, 2.0, (30, 3))])
    depth = t.max_depth
    levels = sorted({0, 1, 2, depth // 2, max(depth - 1, 0), depth, 25})

    def points(offs, pairs, i):
        return {p for f, l in pairs[offs[i]:offs[i + 1]] for p in range(int(f), int(l))}

    for kn, kv in KERNELS.items():
        r = 2.5
        eo, ep, _ = oc.neighborsStruct(q, r, kn)
        for level in levels:
            res = {}
            for upper in (False, True):
                ro, pairs, npts = oc.neighborsApprox(q, r, level, upper, kn)
                o2, p2 = t.approx_ranges(sxyz, kv, q, r, level, upper)
                assert_ranges_equal(ro, pairs, o2, p2, f"{kn} level {level} upper {upper}")
                lens = pairs[:, 1].astype(np.int64) - pairs[:, 0].astype(np.int64)
                csum = np.concatenate([[0], np.cumsum(lens)])
                want = csum[ro[1:].astype(np.int64)] - csum[ro[:-1].astype(np.int64)]
                assert np.array_equal(npts.astype(np.int64), want), "numberOfPoints"
                res[upper] = (ro, pairs)
            for i in range(0, len(q), 23):
                exact = points(eo, ep, i)
                assert points(*res[False], i) <= exact <= points(*res[True], i), f"{kn} level {level} query {i}"
    oc.close()


@pytest.mark.parametrize("case", range(len(SYNTH)))
@pytest.mark.parametrize("search", ["lanes8", "packet", "knn_packet", "knn_packet_fp32", "knn_leaves",
                                    "knn_bucket2k", "packet_fp32_radius", "packet_fp32_knn"])
def test_gpu_knn_matches_oracle(synth_cases, case, search):
    xyz, enc, leaf, keys, perm, box, sxyz, t = synth_cases[case]
    oc = octree(xyz, enc, leaf, search)
    q = sxyz[query_indices(300, len(sxyz), seed=100 + case)]
    # also centres that are not cloud points
    q = np.concatenate([q, q[:50] + np.random.default_rng(case).normal(0, 1.0, (50, 3))])
    for k in (1, 10, 16, 17, 50, 64, 65, 128, 250, 1000):
        idx, d2, cnt = oc.knn(q, k)
        i2, d22, c2 = t.knn(sxyz, q, k)
        assert_knn_equal(idx, d2, cnt, i2, d22, c2, sxyz, q, f"k={k}")
        # the oracle applies the same tie rule: identical arrays
        assert np.array_equal(idx[:, :].astype(np.int64)[d2 < np.inf], i2.astype(np.int64)[d22 < np.inf])
    oc.close()
