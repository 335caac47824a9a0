"""The one-pass packet radius search (result chunks + compaction) against the
two-pass form (count, scan, fill) and the oracle.

Both forms must give the same CSR bit for bit: offsets and every query's
ascending index list, for every kernel and variant, scalar and per-query
radii.  A large radius makes the first pool (3 chunks per query) too small, so
the search sizes the pool from the exact counts and runs again.
"""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.synth import lidar_tile, query_indices
from tests.parity import assert_csr_equal

pytestmark = pytest.mark.gpu

KERNELS = ["sphere", "circle", "cube", "square"]
ALGOS = ["neighborsPrune", "neighbors", "neighborsStruct"]


@pytest.fixture(scope="module")
def cloud():
    oc = LinearOctree(lidar_tile(120_000, 110.0, 61), encoder="hilbert", max_points_leaf=32)
    _, _, sxyz = oc.sorted_points()
    return oc, sxyz


def both(oc, centres, radius, kernel, algo):
    oc.set_search_config(packet=True, two_pass=True)
    two = oc.radius_search(centres, radius, kernel, algo)
    oc.set_search_config(packet=True, two_pass=False)
    one = oc.radius_search(centres, radius, kernel, algo)
    return one, two


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("algo", ALGOS)
def test_one_pass_equals_two_pass(cloud, kernel, algo):
    oc, sxyz = cloud
    c = sxyz[query_indices(3000, len(sxyz), 17)]
    rng = np.random.default_rng(5)
    for radius in (1.7, rng.uniform(0.3, 4.0, len(c))):
        (o1, i1), (o2, i2) = both(oc, c, radius, kernel, algo)
        assert np.array_equal(o1, o2)
        assert np.array_equal(i1, i2)


def test_pool_resize_rerun_matches_oracle(cloud, port):
    oc, sxyz = cloud
    c = sxyz[query_indices(800, len(sxyz), 23)]
    (o1, i1), (o2, i2) = both(oc, c, 12.0, "sphere", "neighborsPrune")  # ~1500 results per query
    assert o1[-1] / len(c) > 3 * 64  # more than the first pool holds
    assert np.array_equal(o1, o2) and np.array_equal(i1, i2)
    keys, _, _ = oc.sorted_points()
    tree = port.build(5, keys, oc.max_points_leaf, oc.box)
    ro, ri = tree.radius(sxyz, 1, 2, c, 12.0)
    assert_csr_equal(o1, i1, ro, ri, "one-pass vs oracle")


def test_one_pass_device_buffers_and_capacity(cloud, torch_cuda):
    """Device-memory calls: a too-small output returns OCT_ERR_CAPACITY with the offsets written."""
    import ctypes as C

    from octrees_benchmark_b200 import capi

    torch = torch_cuda
    oc, sxyz = cloud
    c = sxyz[query_indices(1000, len(sxyz), 29)]
    dc = torch.from_numpy(np.ascontiguousarray(c)).cuda()
    offs = torch.zeros(len(c) + 1, dtype=torch.int64, device="cuda")
    out = torch.zeros(10, dtype=torch.int32, device="cuda")
    tot = C.c_uint64()
    oc.set_search_config(packet=True)
    L = capi.lib()
    st = L.oct_radius_search(oc.handle, 1, 2, dc.data_ptr(), len(c), None, 2.0, offs.data_ptr(), out.data_ptr(), 10,
                             C.byref(tot), capi.OCT_MEM_DEVICE)
    assert st == capi.OCT_ERR_CAPACITY and tot.value > 10
    want_o, want_i = oc.radius_search(c, 2.0, "sphere", "neighborsPrune")
    assert np.array_equal(offs.cpu().numpy().view(np.uint64), want_o)
    out = torch.zeros(tot.value, dtype=torch.int32, device="cuda")
    st = L.oct_radius_search(oc.handle, 1, 2, dc.data_ptr(), len(c), None, 2.0, offs.data_ptr(), out.data_ptr(),
                             tot.value, C.byref(tot), capi.OCT_MEM_DEVICE)
    assert st == capi.OCT_OK
    capi.check(L.oct_synchronize(oc.handle), oc.handle)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want_i)


@pytest.fixture(scope="module")
def torch_cuda():
    return pytest.importorskip("torch")
