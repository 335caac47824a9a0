"""The checker for the Vector-radii overloads (square and cube kernels with
per-axis radii, linear_octree.hpp:1044-1074): the compiled reference's
results equal a brute-force box test over the sorted cloud (closed intervals,
centre -/+ radii per axis, kernel_abstract.hpp:41-45, kernel_3d.hpp:273-283,
kernel_2d.hpp:153-162)."""
import numpy as np
import pytest

from octrees_benchmark_b200.synth import lidar_tile
from tests.parity import csr_set_diffs


@pytest.fixture(scope="module")
def ref():
    from oracle import oracle

    if not oracle.reference_available():
        pytest.skip("oracle/_ref is not built")
    xyz = lidar_tile(30_000, 60.0, seed=7)
    return oracle.Reference(5, xyz, 32)


@pytest.mark.parametrize("kernel", [2, 3])
@pytest.mark.parametrize("algo", [1, 2, 3])
def test_reference_axes_equal_brute_force(ref, kernel, algo):
    sxyz = ref.points()[0]
    rng = np.random.default_rng(3)
    q = sxyz[rng.integers(0, len(sxyz), 200)]
    r3 = rng.uniform(0.3, 4.0, (200, 3))
    offs, idx, _, _ = ref.radius_axes(kernel, algo, q, r3)
    lo, hi = q - r3, q + r3
    dims = 3 if kernel == 3 else 2
    want_o, want_i = [0], []
    for j in range(len(q)):
        m = np.all((sxyz[:, :dims] >= lo[j, :dims]) & (sxyz[:, :dims] <= hi[j, :dims]), axis=1)
        ids = np.nonzero(m)[0]
        want_i.append(ids)
        want_o.append(want_o[-1] + len(ids))
    assert csr_set_diffs(offs, idx, np.array(want_o), np.concatenate(want_i)) == 0
    assert int(offs[-1]) > len(q)
