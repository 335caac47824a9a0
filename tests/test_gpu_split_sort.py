"""The split sort (four passes over the upper key halves, then the runs of
equal upper halves by their full keys) against the oracle's stable sort and
against the cloud's 8-pass sort (OCT_CLOUD_SORT_8PASS): keys, permutation,
sorted points and the tree arrays bitwise.  The clouds exercise every run
path: short runs (the synthetic tile), runs of 33..4096 points (dense
clusters, sorted in shared memory), and runs above 4096 points (clusters of
thousands of points in one cell: one such run, and 300 of them, which takes
two bytes of run slot in the long-run stage's keys)."""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.synth import lidar_tile
from tests.parity import same_f64

pytestmark = pytest.mark.gpu


def clustered(n_tile, clusters, seed):
    """A tile plus clusters of (size, spread in metres) around random tile points; exact duplicates too."""
    rng = np.random.default_rng(seed)
    xyz = lidar_tile(n_tile, 200.0, seed)
    parts = [xyz]
    for size, spread in clusters:
        c = xyz[rng.integers(0, n_tile)]
        parts.append(c + rng.normal(0.0, spread, (size, 3)) if spread > 0 else np.repeat(c[None], size, 0))
    out = np.concatenate(parts)
    return out[rng.permutation(len(out))]


CASES = {
    "tile": clustered(300_000, [], 1),
    "mid_runs": clustered(200_000, [(40, 1e-7), (300, 1e-7), (1500, 1e-8), (4000, 1e-9), (700, 0.0)], 2),
    "long_run": clustered(100_000, [(6000, 1e-9), (200, 1e-7)], 3),
    "many_long_runs": clustered(60_000, [(4100 + 7 * j, 1e-9 if j % 3 else 0.0) for j in range(300)], 4),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("enc", [1, 5])
def test_split_sort_equals_oracle_and_8pass(port, case, enc):
    xyz = CASES[case]
    keys, perm, box, sxyz = port.encode_sort(enc, xyz)
    a = LinearOctree(xyz, encoder=enc, max_points_leaf=32)
    b = LinearOctree(xyz, encoder=enc, max_points_leaf=32, sort_8pass=True)
    for oc in (a, b):
        gk, gp, gx = oc.sorted_points()
        assert np.array_equal(gk, keys)
        assert np.array_equal(gp.astype(np.uint64), np.asarray(perm, np.uint64))
        assert same_f64(gx, sxyz)
        assert same_f64(oc.box, box)
    ea, eb = a.export(), b.export()
    for k in ("offsets", "ranges"):
        assert np.array_equal(ea[k], eb[k])
    assert same_f64(ea["centers"], eb["centers"])
    a.close()
    b.close()


def test_split_sort_repeated_builds(port):
    """The same cloud object sorted again after new points (scratch from the previous sort left behind)."""
    oc = LinearOctree(CASES["mid_runs"], encoder=5, max_points_leaf=64)
    for case in ("long_run", "tile", "mid_runs"):
        xyz = CASES[case]
        keys, perm, box, sxyz = port.encode_sort(5, xyz)
        from octrees_benchmark_b200 import capi
        import ctypes as C

        L = capi.lib()
        capi.check(L.oct_set_points(oc.handle, np.ascontiguousarray(xyz).ctypes.data, len(xyz), 0), oc.handle)
        box12 = np.zeros(12)
        gk = np.zeros(len(xyz), np.uint64)
        gp = np.zeros(len(xyz), np.uint32)
        capi.check(L.oct_encode_sort(oc.handle, box12.ctypes.data, gk.ctypes.data, gp.ctypes.data, None, 0),
                   oc.handle)
        assert np.array_equal(gk, keys) and np.array_equal(gp.astype(np.uint64), np.asarray(perm, np.uint64))
        assert same_f64(box12, box)
        info = capi.OctTreeInfo()
        capi.check(L.oct_build(oc.handle, C.byref(info)), oc.handle)
    oc.close()
