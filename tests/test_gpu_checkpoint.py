"""Checkpoints (oct_tree_import): a built cloud saved with np.savez and restored
without sorting or building answers every search bitwise as the original does,
on the packet, plain and FP32-filter paths and in an engine batch; corrupted
checkpoints are rejected before anything is uploaded."""
import numpy as np
import pytest

from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.capi import OctError
from octrees_benchmark_b200.synth import lidar_tile, query_indices

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def saved(tmp_path_factory):
    oc = LinearOctree(lidar_tile(50_000, 80.0, 17), encoder="hilbert", max_points_leaf=32)
    path = tmp_path_factory.mktemp("ck") / "cloud.npz"
    np.savez(path, **oc.checkpoint())
    return oc, path


def searches(oc, q):
    out = [oc.radius_search(q, 2.0, "sphere", "neighborsPrune"), oc.radius_search(q, 1.5, "cube", "neighbors"),
           oc.neighborsStruct(q, 2.0, "circle"), oc.neighborsApprox(q, 2.0, 3, True, "sphere"),
           oc.neighborsApprox(q, 2.0, 3, False, "sphere"), oc.knn(q, 10), oc.knn(q, 50), oc.knn(q, 200)]
    return [a for res in out for a in res]


@pytest.mark.parametrize("path_cfg", [dict(packet=True), dict(packet=False), dict(packet=True, fp32_filter=True)])
def test_restored_cloud_answers_like_the_original(saved, path_cfg):
    oc, path = saved
    with np.load(path) as z:
        rc = LinearOctree.from_checkpoint({k: z[k] for k in z.files}, **path_cfg)
    oc.set_search_config(**path_cfg)
    for a, b in zip(oc.sorted_points(), rc.sorted_points()):
        assert np.array_equal(a, b)
    for k, v in oc.export().items():
        assert np.array_equal(v, rc.export()[k]), k
    assert (rc.n_leaf, rc.n_internal, rc.n_total, rc.max_depth_seen) == (oc.n_leaf, oc.n_internal, oc.n_total,
                                                                         oc.max_depth_seen)
    _, _, sxyz = oc.sorted_points()
    q = np.concatenate([sxyz[query_indices(700, len(sxyz), seed=4)], sxyz[:50] + 1.7])
    for a, b in zip(searches(oc, q), searches(rc, q)):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    oc.set_search_config()
    rc.close()


def test_restored_cloud_in_an_engine_batch(saved):
    torch = pytest.importorskip("torch")
    from octrees_benchmark_b200.engine import BatchEngine, Request

    oc, path = saved
    with np.load(path) as z:
        rc = LinearOctree.from_checkpoint({k: z[k] for k in z.files})
    _, _, sxyz = oc.sorted_points()
    q = torch.from_numpy(np.ascontiguousarray(sxyz[query_indices(900, len(sxyz), seed=5)])).cuda()
    res = []
    for cloud in (oc, rc):
        eng = BatchEngine()
        pl = eng.run([Request(cloud, "radius", q, radius=2.0, kernel="sphere", algo="neighborsPrune"),
                      Request(cloud, "knn", q, k=20)])
        res.append([*eng.radius_result(pl[0]), *eng.knn_result(pl[1], 20)])
    for a, b in zip(*res):
        assert np.array_equal(a, b)
    rc.close()


@pytest.mark.parametrize("damage", ["keys", "perm", "offsets", "ranges", "counts"])
def test_corrupted_checkpoint_is_rejected(saved, damage):
    oc, _ = saved
    ck = oc.checkpoint()
    if damage == "keys":
        ck["keys"] = ck["keys"].copy()
        ck["keys"][[10, 11]] = ck["keys"][[11, 10]] + np.array([1, 0], np.uint64)  # out of order
    elif damage == "perm":
        ck["perm"] = ck["perm"].copy()
        ck["perm"][5] = ck["perm"][6]
    elif damage == "offsets":
        ck["offsets"] = ck["offsets"].copy()
        ck["offsets"][0] = np.uint32(ck["info"][3])  # first child past the last node
    elif damage == "ranges":
        ck["ranges"] = ck["ranges"].copy()
        ck["ranges"][3, 1] = np.uint64(ck["info"][0] + 1)
    else:
        ck["info"] = ck["info"].copy()
        ck["info"][2] += 1
    with pytest.raises(OctError):
        LinearOctree.from_checkpoint(ck)
