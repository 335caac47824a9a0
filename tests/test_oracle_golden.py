"""Pin the CPU oracle (oracle/octree_oracle.c) before trusting it.

1. Against the golden fixtures written by the UNMODIFIED reference
   (tests/golden/make_golden.py): keys, ids, Box, tree arrays, every radius
   kernel x variant, neighborsStruct ranges, kNN, anchor-coordinate edge cases
   and Morton / Hilbert key tables.
2. Against the known answers of the reference's own GoogleTest suite
   (tests/structures/test_octree.cpp, test_octree_advanced.cpp,
   tests/integration/test_complex.cpp, tests/encoding/test_encoders.cpp),
   restated here.
"""
import glob
import os

import numpy as np
import pytest

from tests.parity import assert_csr_equal, assert_knn_equal, assert_ranges_equal, same_f64, sq_dist

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CLOUDS = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz")) if not p.endswith("keys_anchor.npz"))
KERNELS = {"sphere": 1, "circle": 0, "cube": 3, "square": 2}


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("path", CLOUDS, ids=[os.path.basename(p)[:-4] for p in CLOUDS])
def test_oracle_matches_golden_cloud(port, path):
    g = load(path)
    enc, leaf = int(g["encoder"]), int(g["max_leaf"])
    keys, perm, box, sxyz = port.encode_sort(enc, g["xyz"])
    assert same_f64(box, g["box"])
    assert np.array_equal(keys, g["keys"])
    assert np.array_equal(perm.astype(np.uint64), g["ids"])
    assert same_f64(sxyz, g["sorted_xyz"])
    t = port.build(enc, keys, leaf, box)
    assert [t.n, t.n_leaf, t.n_internal, t.n_total, t.max_depth] == [int(v) for v in g["info"]]
    arr = t.arrays()
    for k in ("offsets", "ranges"):
        assert np.array_equal(arr[k], g["tree_" + k]), k
    for k in ("centers", "radii", "half"):
        assert same_f64(arr[k], g["tree_" + k]), k
    q = g["centers"]
    for ri, r in enumerate(g["radii"]):
        for kn, kv in KERNELS.items():
            for algo in (1, 2, 3):
                offs, idx = t.radius(sxyz, kv, algo, q, r)
                assert_csr_equal(offs, idx, g[f"rad_{ri}_{kn}_{algo}_offs"], g[f"rad_{ri}_{kn}_{algo}_idx"],
                                 f"{kn} algo {algo} r {r}")
            offs, pairs = t.struct_ranges(sxyz, kv, q, r)
            assert_ranges_equal(offs, pairs, g[f"struct_{ri}_{kn}_offs"], g[f"struct_{ri}_{kn}_pairs"], kn)
    for k in g["ks"]:
        k = int(k)
        idx, d2, cnt = t.knn(sxyz, q, k)
        assert_knn_equal(idx, d2, cnt, g[f"knn_{k}_idx"], g[f"knn_{k}_d2"], g[f"knn_{k}_cnt"], sxyz, q, f"k={k}")


def test_oracle_anchor_and_key_tables(port):
    g = load(os.path.join(GOLDEN, "keys_anchor.npz"))
    got = np.array([port.anchor(*t) for t in g["pcr"]], np.uint64)
    assert np.array_equal(got, g["anchors"])
    for enc, name in ((1, "morton"), (5, "hilbert")):
        keys = np.array([port.encode_xyz(enc, *map(int, c)) for c in g["coords"]], np.uint64)
        assert np.array_equal(keys, g[name])
        dec = np.array([port.decode_key(enc, int(k)) for k in keys], np.uint64)
        assert np.array_equal(dec, g[name + "_dec"])


# ---- the reference's own known-answer tests, restated against the oracle ----

def _tree(port, pts, enc=1, leaf=128):
    keys, perm, box, sxyz = port.encode_sort(enc, np.asarray(pts, np.float64).reshape(-1, 3))
    return port.build(enc, keys, leaf, box), sxyz, box


def test_reference_octree_knn_and_square(port):
    # test_octree.cpp:17-80: eight points in three clusters
    pts = [[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0], [10, 10, 10], [10.1, 10, 10], [10, 10.1, 10], [5, 5, 5],
           [5, 5, 5.1]]
    t, sxyz, _ = _tree(port, pts)
    idx, d2, cnt = t.knn(sxyz, np.array([[9.9, 9.9, 9.9]]), 2)
    assert abs(d2[0, 0] - 0.03) < 1e-4
    assert sxyz[idx[0, 0], 0] > 9.0
    offs, ids = t.radius(sxyz, 2, 2, np.array([[5.0, 5.0, 5.0]]), 0.25)
    assert len(ids) == 2
    assert sorted(sxyz[ids, 2]) == [5.0, 5.1]


def test_reference_advanced_cases(port):
    # test_octree_advanced.cpp:33-131
    t, sxyz, _ = _tree(port, np.zeros((0, 3)))                       # empty cloud
    offs, ids = t.radius(sxyz, 2, 2, np.zeros((1, 3)), 1.0)
    assert len(ids) == 0
    idx, d2, cnt = t.knn(sxyz, np.zeros((1, 3)), 1)
    assert cnt[0] == 0
    t, sxyz, _ = _tree(port, [[1, 1, 1], [1, 1, 1], [2, 2, 2]])        # duplicates
    idx, d2, cnt = t.knn(sxyz, np.array([[1.0, 1.0, 1.0]]), 5)
    assert cnt[0] == 3 and d2[0, 0] == 0.0 and d2[0, 1] == 0.0 and abs(d2[0, 2] - 3.0) < 1e-9
    t, sxyz, _ = _tree(port, [[0, 0, 0], [0, 0, 0], [1, 1, 1]])        # zero radius
    offs, ids = t.radius(sxyz, 2, 2, np.zeros((1, 3)), 0.0)
    assert len(ids) == 2
    t, sxyz, _ = _tree(port, [[0, 0, 0], [10, 10, 10], [5, 5, 5]])     # boundary
    offs, ids = t.radius(sxyz, 2, 2, np.array([[10.0, 10.0, 10.0]]), 0.0)
    assert len(ids) == 1
    offs, ids = t.radius(sxyz, 2, 2, np.array([[10.1, 10.1, 10.1]]), 0.01)
    assert len(ids) == 0
    t, sxyz, _ = _tree(port, [[1, 1, 1], [2, 0, 0]])                  # sphere
    assert len(t.radius(sxyz, 1, 2, np.zeros((1, 3)), 1.5)[1]) == 0
    assert len(t.radius(sxyz, 1, 2, np.zeros((1, 3)), 2.5)[1]) == 2
    t, sxyz, _ = _tree(port, [[1, 1, 1], [2, 2, 2]])                  # cube
    offs, ids = t.radius(sxyz, 3, 2, np.zeros((1, 3)), 1.5)
    assert len(ids) == 1 and sxyz[ids[0], 0] == 1.0


def test_reference_complex_cases(port):
    # test_complex.cpp:37-114: brute force by count (<=), degenerate line / plane, large offsets
    def brute(xyz, c, r):
        return int(np.sum(sq_dist(xyz, c) <= r * r))

    line = np.stack([np.arange(100) * 0.1, np.zeros(100), np.zeros(100)], 1)
    t, sxyz, _ = _tree(port, line)
    c = np.array([5.0, 0.0, 0.0])
    assert len(t.radius(sxyz, 1, 2, c[None], 0.55)[1]) == brute(sxyz, c, 0.55)
    g = np.stack(np.meshgrid(np.arange(10) * 0.1, np.arange(10) * 0.1, indexing="ij"), -1).reshape(-1, 2)
    plane = np.concatenate([g, np.zeros((100, 1))], 1)
    t, sxyz, _ = _tree(port, plane)
    c = np.array([0.5, 0.5, 0.0])
    assert len(t.radius(sxyz, 1, 2, c[None], 0.2)[1]) == brute(sxyz, c, 0.2)
    o = 1e6
    t, sxyz, _ = _tree(port, [[o, o, o], [o + 0.1, o, o], [o, o + 0.1, o]])
    assert len(t.radius(sxyz, 1, 2, np.array([[o + 0.05, o + 0.05, o]]), 0.1)[1]) == 3
    k = port.encode_xyz(1, 1000, 2000, 3000)
    assert port.decode_key(1, k) == (1000, 2000, 3000)


def test_reference_encoder_sorting(port):
    # test_encoders.cpp:29-64: four points, (1,1,1) first and (9,9,9) last under Morton
    pts = np.array([[1, 1, 1], [9, 9, 9], [5, 5, 5], [1, 9, 1]], np.float64)
    keys, perm, box, sxyz = port.encode_sort(1, pts)
    assert list(sxyz[0]) == [1, 1, 1] and list(sxyz[3]) == [9, 9, 9]
    for enc in (1, 5):
        _, _, box, _ = port.encode_sort(enc, pts)
        assert box[6] == 1.0 and box[9] == 9.0 and box[7] == 1.0 and box[10] == 9.0


def test_reference_knn_consistency(port):
    # test_complex.cpp:144-173: ascending distances that match a recomputation
    rng = np.random.default_rng(42)
    pts = rng.uniform(0, 10, (500, 3))
    t, sxyz, _ = _tree(port, pts)
    c = np.array([[5.0, 5.0, 5.0]])
    idx, d2, cnt = t.knn(sxyz, c, 10)
    assert np.all(np.diff(d2[0]) >= 0)
    assert np.allclose(d2[0], sq_dist(sxyz[idx[0].astype(np.int64)], c[0]), atol=1e-7)
