"""The oracle against the compiled reference (oracle/_ref) on larger seeded
clouds than the fixtures hold.  Skipped where oracle/_ref was not built (it is
built from the reference sources by ``make -C oracle ref``)."""
import numpy as np
import pytest

from octrees_benchmark_b200.synth import lidar_tile, query_indices
from oracle.oracle import Reference, reference_available
from tests.parity import assert_csr_equal, assert_knn_equal, assert_ranges_equal, same_f64

pytestmark = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")

CASES = [
    # (n, tile, seed, encoder, leaf)
    (60_000, 120.0, 21, 1, 64),
    (60_000, 120.0, 22, 5, 128),
    (8_000, 40.0, 23, 5, 1),     # deep tree: every point in its own leaf down to level 21 for duplicates
    (20_000, 60.0, 24, 1, 7),
]


@pytest.mark.parametrize("n,tile,seed,enc,leaf", CASES)
def test_oracle_equals_reference(port, n, tile, seed, enc, leaf):
    xyz = lidar_tile(n, tile, seed)
    if seed == 23:
        xyz[::7] = xyz[3]  # many exact duplicates
    R = Reference(enc, xyz, leaf)
    rxyz, rids, rkeys = R.points()
    keys, perm, box, sxyz = port.encode_sort(enc, xyz)
    assert same_f64(box, R.box())
    assert np.array_equal(keys, rkeys)
    assert np.array_equal(perm.astype(np.uint64), rids)
    t = port.build(enc, keys, leaf, box)
    assert (t.n_leaf, t.n_internal, t.n_total, t.max_depth) == (R.n_leaf, R.n_internal, R.n_total, R.max_depth)
    a, b = t.arrays(), R.arrays()
    for k in a:
        assert same_f64(a[k], b[k]) if a[k].dtype == np.float64 else np.array_equal(a[k], b[k]), k
    q = sxyz[query_indices(200, n, seed=seed)]
    for kern in range(4):
        for algo in (1, 2, 3):
            for r in (0.3, 1.5, 4.0):
                o1, i1 = t.radius(sxyz, kern, algo, q, r)
                o2, i2 = R.radius(kern, algo, q, r)
                # the oracle reproduces even the reference's emission order
                assert np.array_equal(o1, o2) and np.array_equal(i1, i2), (kern, algo, r)
        o1, p1 = t.struct_ranges(sxyz, kern, q, 1.5)
        o2, p2 = R.struct_ranges(kern, q, 1.5)
        assert_ranges_equal(o1, p1, o2, p2)
        # neighborsApprox through the reference's public overload (percentage -> level)
        for level in sorted({0, 2, t.max_depth // 2, t.max_depth, 21}):
            for upper in (False, True):
                o1, p1 = t.approx_ranges(sxyz, kern, q, 1.5, level, upper)
                o2, p2 = R.approx_ranges(kern, q, 1.5, float(level), upper)
                assert np.array_equal(o1, o2) and np.array_equal(p1, p2), (kern, level, upper)
    for k in (1, 10, 50):
        i1, d1, c1 = t.knn(sxyz, q, k)
        i2, d2, c2 = R.knn(q, k)
        assert_knn_equal(i1, d1, c1, i2, d2, c2, sxyz, q, f"k={k}", lowest_ties=False)


def test_anchor_edge_cases_against_reference(port):
    vals = [(0, 0, 0), (1, 1, 0), (-1.5, 0, 1), (np.nan, 0, 1), (np.inf, 0, 1), (-np.inf, 0, 1), (2.0, 0.0, 1.0),
            (0.9999999999999999, 0, 0.5), (-1e-300, 0, 1e-300)]
    for p, c, r in vals:
        assert port.anchor(p, c, r) == Reference.anchor(p, c, r), (p, c, r)
