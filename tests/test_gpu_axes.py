"""The Vector-radii overloads on the device (oct_radius_search_axes /
oct_struct_search_axes): square and cube kernels with per-axis radii, one
vector per query or one for all, neighbors / neighborsPrune / neighborsStruct,
against the compiled reference (linear_octree.hpp:1044-1074,
kernel_factory.hpp:33-41).  Other kernels are rejected as the reference's
static_assert rejects them."""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree, capi
from octrees_benchmark_b200.synth import lidar_tile
from tests.parity import csr_set_diffs, ranges_diffs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(1, 16), (5, 64)], ids=["morton16", "hilbert64"])
def clouds(request):
    from oracle import oracle

    if not oracle.reference_available():
        pytest.skip("oracle/_ref is not built")
    enc, leaf = request.param
    xyz = lidar_tile(150_000, 120.0, seed=11)
    R = oracle.Reference(enc, xyz, leaf)
    oc = LinearOctree(xyz, encoder=enc, max_points_leaf=leaf)
    yield oc, R
    oc.close()


@pytest.mark.parametrize("kernel", ["square", "cube"])
@pytest.mark.parametrize("per_query", [True, False], ids=["per_query", "one_vector"])
def test_axes_match_reference(clouds, kernel, per_query):
    oc, R = clouds
    sxyz = R.points()[0]
    rng = np.random.default_rng(5)
    q = sxyz[rng.integers(0, len(sxyz), 3000)]
    r3 = rng.uniform(0.2, 5.0, (3000, 3)) if per_query else np.array([0.7, 3.3, 1.9])
    kv = capi.KERNELS[kernel]
    for algo in ("neighbors", "neighborsPrune", "neighborsStruct"):
        ro, ri, rso, rsp = R.radius_axes(kv, capi.ALGOS[algo], q, r3)
        offs, idx = oc.radius_search_axes(q, r3, kernel, algo)
        assert csr_set_diffs(offs, idx, ro, ri) == 0, f"{kernel} {algo}"
        assert int(offs[-1]) > len(q)
    go, gp, npts = oc.neighborsStruct_axes(q, r3, kernel)
    assert ranges_diffs(go, gp, rso, rsp) == 0
    assert np.array_equal(npts, np.diff(ro.astype(np.int64)))


def test_axes_reject_round_kernels(clouds):
    oc, _ = clouds
    q = np.zeros((4, 3))
    for kernel in ("sphere", "circle"):
        with pytest.raises(capi.OctError) as ei:
            oc.radius_search_axes(q, np.array([1.0, 1.0, 1.0]), kernel, "neighborsPrune")
        assert ei.value.status == capi.OCT_ERR_INVALID_ARG
