"""The kNN provisional threshold (packet path) changes no result.

With the estimate on (default and a small factor that often undershoots), off,
the returned indices, squared distances and counts are identical, for centres
at cloud points, off the cloud (above the terrain, outside the tile: the
estimate finds fewer than k points and the query runs again) and for a cloud
with fewer than k points.  Both kNN kernels of the packet path are covered:
one warp per query (register lists) and groups of queries per warp, whose
undershooting queries go to the fallback list.  One case of each is also
checked against the oracle.
"""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.synth import lidar_tile, query_indices
from tests.parity import assert_knn_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cloud():
    oc = LinearOctree(lidar_tile(80_000, 90.0, 71), encoder="hilbert", max_points_leaf=64)
    _, _, sxyz = oc.sorted_points()
    return oc, sxyz


def centres(sxyz):
    rng = np.random.default_rng(3)
    at = sxyz[query_indices(1500, len(sxyz), 5)]
    above = at + np.array([0.0, 0.0, 30.0])
    outside = rng.uniform(-200.0, 300.0, (300, 3))
    return np.concatenate([at, above, outside])


@pytest.mark.parametrize("group", [False, True])
@pytest.mark.parametrize("k", [1, 10, 33, 50, 64])
def test_estimate_on_off_identical(cloud, k, group):
    oc, sxyz = cloud
    c = centres(sxyz)
    res = []
    for est in (0, 30, -1):
        oc.set_search_config(packet=True, knn_packet=group, knn_estimate=est)
        res.append(oc.knn(c, k))
    oc.set_search_config(packet=True, knn_packet=not group, knn_estimate=0)
    res.append(oc.knn(c, k))
    for r in res[1:]:
        for a, b in zip(res[0], r):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("group", [False, True])
def test_estimate_matches_oracle(cloud, port, group):
    oc, sxyz = cloud
    c = centres(sxyz)[::7]
    oc.set_search_config(packet=True, knn_packet=group, knn_estimate=0)
    idx, d2, cnt = oc.knn(c, 50)
    keys, _, _ = oc.sorted_points()
    tree = port.build(5, keys, oc.max_points_leaf, oc.box)
    oi, od, ocnt = tree.knn(sxyz, c, 50)
    assert_knn_equal(idx, d2, cnt, oi, od, ocnt, sxyz, c, "kNN with the estimate vs oracle")


@pytest.mark.parametrize("group", [False, True])
def test_cloud_smaller_than_k(group):
    oc = LinearOctree(lidar_tile(40, 10.0, 72), encoder="morton", max_points_leaf=8)
    c = lidar_tile(40, 10.0, 72)[:10]
    oc.set_search_config(packet=True, knn_packet=group, knn_estimate=0)
    a = oc.knn(c, 64)
    oc.set_search_config(packet=True, knn_packet=group, knn_estimate=-1)
    b = oc.knn(c, 64)
    assert (a[2] == 40).all()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
