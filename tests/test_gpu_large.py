"""The large skewed cloud at full size against the compiled reference (opt-in:
the reference's copy of the cloud holds tens of GB of host memory and the
run takes about a minute (53 s on a B200 machine with 196 GB of RAM), so it runs only with
OCT_LARGE=1, e.g. `OCT_LARGE=1 python -m pytest tests/test_gpu_large.py -m gpu`).

500,000,000 points on a 10 km tile (seed 3, generated on the device: rural
ground at 5 pts/m^2 plus 50 urban building clusters at ~2000 pts/m^2), Hilbert,
leaf 64.  The reference builds the same cloud on the host cores; the Box, the
tree sizes and depth must be equal, and on a sample of 10,000 radius centres
(sphere, neighborsPrune, r = 2.5 m, FP32 filter + FP64 band) and 10,000 kNN
centres (k = 1000, the list kernel) at SearchSet positions every neighbour set
and every kNN result must equal the reference's (d^2 bitwise, ties by lowest
index)."""
import os

import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.synth import large_tile_device, search_set
from tests.parity import csr_set_diffs, knn_diffs, same_f64

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("OCT_LARGE") != "1", reason="opt-in: set OCT_LARGE=1")]

N = int(os.environ.get("OCT_LARGE_POINTS", "500000000"))


def test_large_cloud_sample_equals_reference():
    torch = pytest.importorskip("torch")
    from oracle import oracle

    if not oracle.reference_available():
        pytest.skip("oracle/_ref is not built")
    xyz_d = large_tile_device(N)
    oc = LinearOctree(xyz_d, encoder=5, max_points_leaf=64, fp32_filter=True)
    xyz_h = xyz_d.cpu().numpy()
    del xyz_d
    torch.cuda.empty_cache()
    R = oracle.Reference(5, xyz_h, 64)
    del xyz_h
    assert same_f64(oc.box, R.box())
    assert (oc.n_leaf, oc.n_internal, oc.n_total, oc.max_depth_seen) == \
        (R.n_leaf, R.n_internal, R.n_total, R.max_depth)
    # sample centres: sorted cloud points at SearchSet positions
    sel = search_set(20_000, N)
    from octrees_benchmark_b200 import capi
    import ctypes as C

    sorted_d = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    capi.check(capi.lib().oct_encode_sort(oc.handle, None, None, None, sorted_d.data_ptr(), capi.OCT_MEM_DEVICE),
               oc.handle)
    capi.check(capi.lib().oct_synchronize(oc.handle), oc.handle)
    q = sorted_d[torch.from_numpy(sel).cuda()].cpu().numpy()
    del sorted_d
    torch.cuda.empty_cache()
    qr, qk = q[:10_000], q[10_000:]
    go, gi = oc.radius_search(qr, 2.5, "sphere", "neighborsPrune")
    ro, ri = R.radius(1, 2, qr, 2.5)
    assert csr_set_diffs(go, gi, ro, ri) == 0
    assert int(ro[-1]) > 10_000
    oc.set_search_config(packet=True, fp32_filter=True)
    ki, kd, kc = oc.knn(qk, 1000)
    rki, rkd, rkc = R.knn(qk, 1000)
    # the sorted cloud on the host only for brute-force tie checks (few rows)
    xyz_sorted = R.points()[0]
    diffs, err, _ = knn_diffs(ki, kd, kc, rki, rkd, rkc, xyz_sorted, qk)
    assert diffs == 0 and err == 0.0
