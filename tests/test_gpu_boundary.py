"""The rest of the drop-in boundary: an octree over a cloud that sortPoints
already ordered (the reference's LinearOctree(points, codes, box, enc),
linear_octree.hpp:614-623, through oct_set_sorted_points) equals the one the
library sorts itself, array for array and search for search; bad codes are
rejected."""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.synth import lidar_tile, query_indices
from tests.parity import assert_csr_equal, assert_knn_equal, same_f64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("enc,leaf", [("morton", 32), ("hilbert", 64)])
def test_from_sorted_equals_one_step(enc, leaf):
    xyz = lidar_tile(120_000, 100.0, seed=17)
    a = LinearOctree(xyz, encoder=enc, max_points_leaf=leaf)
    keys, perm, sxyz = a.sorted_points()
    b = LinearOctree.from_sorted(sxyz, keys, a.box, encoder=enc, max_points_leaf=leaf)
    assert (a.n_total, a.n_leaf, a.max_depth_seen) == (b.n_total, b.n_leaf, b.max_depth_seen)
    ea, eb = a.export(), b.export()
    for k in ("offsets", "ranges"):
        assert np.array_equal(ea[k], eb[k]), k
    for k in ("centers", "radii", "half"):
        assert same_f64(ea[k], eb[k]), k
    kb, pb, xb = b.sorted_points()
    assert np.array_equal(kb, keys) and same_f64(xb, sxyz) and np.array_equal(pb, np.arange(len(keys)))
    q = sxyz[query_indices(2000, len(sxyz), 9)]
    for kern in ("sphere", "cube"):
        oa, ia = a.radius_search(q, 2.0, kern, "neighborsPrune")
        ob, ib = b.radius_search(q, 2.0, kern, "neighborsPrune")
        assert_csr_equal(oa, ia, ob, ib, kern)
    i1, d1, c1 = a.knn(q, 20)
    i2, d2, c2 = b.knn(q, 20)
    assert_knn_equal(i2, d2, c2, i1, d1, c1, sxyz, q, "k=20")
    a.close()
    b.close()


def test_from_sorted_rejects_bad_codes():
    xyz = lidar_tile(5_000, 30.0, seed=18)
    a = LinearOctree(xyz, encoder="hilbert", max_points_leaf=32)
    keys, _, sxyz = a.sorted_points()
    bad = keys.copy()
    bad[11] = bad[10] - np.uint64(1)  # descending
    with pytest.raises(capi.OctError) as ei:
        LinearOctree.from_sorted(sxyz, bad, a.box, encoder="hilbert", max_points_leaf=32)
    assert ei.value.status == capi.OCT_ERR_INVALID_ARG
    top = keys.copy()
    top[-1] = np.uint64(1) << np.uint64(63)
    with pytest.raises(capi.OctError) as ei:
        LinearOctree.from_sorted(sxyz, top, a.box, encoder="hilbert", max_points_leaf=32)
    assert ei.value.status == capi.OCT_ERR_INVALID_ARG
    a.close()
