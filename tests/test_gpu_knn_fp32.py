"""The group kNN's FP32 filter (k <= 64, packet path, fp32_filter on) changes
no result: the same indices, squared distances and counts as the FP64 walk,
for centres at cloud points, above the terrain and outside the tile, on a tile
far from the origin (UTM-sized coordinates, where FP32 keeps the fewest digits)
and with the provisional threshold on and off; the filter's counters show the
FP32 tests, the FP64 tests they leave, and band hits below the FP64 tests."""
import ctypes as C

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.synth import lidar_tile, query_indices
from tests.parity import assert_knn_equal

pytestmark = pytest.mark.gpu


def centres(sxyz, seed):
    rng = np.random.default_rng(seed)
    at = sxyz[query_indices(1200, len(sxyz), seed)]
    lo, hi = sxyz.min(0), sxyz.max(0)
    return np.concatenate([at, at[:200] + np.array([0.0, 0.0, 25.0]),
                           rng.uniform(lo - 50.0, hi + 50.0, (200, 3))])


@pytest.mark.parametrize("offset", [0.0, 4.6e6])
@pytest.mark.parametrize("k", [1, 16, 50, 64])
def test_fp32_filter_identical(offset, k):
    xyz = lidar_tile(60_000, 120.0, 81)
    xyz[:, :2] += offset
    oc = LinearOctree(xyz, encoder="hilbert", max_points_leaf=64)
    _, _, sxyz = oc.sorted_points()
    c = centres(sxyz, 4)
    res = {}
    for fp32 in (0, capi.OCT_FP32_ALL, capi.OCT_FP32_KNN, capi.OCT_FP32_RADIUS):
        for est in (0, -1):
            oc.set_search_config(packet=True, fp32_filter=fp32, knn_packet=True, knn_estimate=est)
            res[(fp32, est)] = oc.knn(c, k)
    base = res[(0, 0)]
    for key, r in res.items():
        for a, b in zip(base, r):
            assert np.array_equal(a, b), key
    oc.close()


def test_fp32_filter_matches_oracle_and_counts(port):
    xyz = lidar_tile(50_000, 100.0, 82)
    oc = LinearOctree(xyz, encoder="morton", max_points_leaf=32)
    _, _, sxyz = oc.sorted_points()
    c = centres(sxyz, 5)[::3]
    oc.set_search_config(packet=True, fp32_filter=True, knn_packet=True)
    L = capi.lib()
    tests, f64, band = C.c_uint64(), C.c_uint64(), C.c_uint64()
    L.oct_knn_filter_stats(oc.handle, None, None, None, 1)
    idx, d2, cnt = oc.knn(c, 50)
    capi.check(L.oct_knn_filter_stats(oc.handle, C.byref(tests), C.byref(f64), C.byref(band), 1), oc.handle)
    keys, _, _ = oc.sorted_points()
    tree = port.build(1, keys, oc.max_points_leaf, oc.box)
    oi, od, ocnt = tree.knn(sxyz, c, 50)
    assert_knn_equal(idx, d2, cnt, oi, od, ocnt, sxyz, c, "FP32-filtered kNN vs oracle")
    assert tests.value > 0 and 0 < f64.value < tests.value and band.value <= f64.value
    oc.close()
