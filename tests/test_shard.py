"""Query sharding across ranks (octrees_benchmark_b200/shard.py) on CPU:
world_size 2 over gloo.  Every rank answers its slice of the queries on its
own replica (the oracle's CPU tree stands in for a GPU replica here: this
checks the split and the gather, not the search) and the gathered CSR and kNN
results equal the one-rank answer."""
import os

import numpy as np
import pytest

from octrees_benchmark_b200.shard import shard_bounds


def test_shard_bounds_cover_and_balance():
    for n in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            parts = [shard_bounds(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [e - b for b, e in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def _rank_main(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    from octrees_benchmark_b200.shard import gather_csr, gather_rows, shard_bounds
    from octrees_benchmark_b200.synth import lidar_tile, query_indices
    from oracle.oracle import Port

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = Port()
        xyz = lidar_tile(20_000, 60.0, seed=31)
        keys, perm, box, sxyz = P.encode_sort(5, xyz)
        tree = P.build(5, keys, 32, box)
        q = sxyz[query_indices(1001, len(sxyz), 4)]
        b, e = shard_bounds(len(q), world, rank)
        offs, idx = tree.radius(sxyz, 1, 2, q[b:e], 2.0)
        go, gi = gather_csr(torch.from_numpy(offs.astype(np.int64)), torch.from_numpy(idx.astype(np.int64)))
        ki, kd, kc = tree.knn(sxyz, q[b:e], 12)
        gki, gkd, gkc = gather_rows(torch.from_numpy(ki.astype(np.int64)), torch.from_numpy(kd),
                                    torch.from_numpy(kc.astype(np.int64)))
        if rank == 0:
            fo, fi = tree.radius(sxyz, 1, 2, q, 2.0)
            fki, fkd, fkc = tree.knn(sxyz, q, 12)
            ok = (np.array_equal(go.numpy(), fo.astype(np.int64)) and np.array_equal(gi.numpy(), fi.astype(np.int64))
                  and np.array_equal(gki.numpy(), fki.astype(np.int64)) and np.array_equal(gkd.numpy(), fkd)
                  and np.array_equal(gkc.numpy(), fkc.astype(np.int64)))
            with open(out_path, "w") as f:
                f.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_equals_one_rank(tmp_path):
    torch = pytest.importorskip("torch")
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "result.txt")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert open(out).read() == "ok"


def _checkpoint_like(seed):
    """A dict with a checkpoint's names and dtypes (0-d scalars, an empty array, 2-D arrays)."""
    rng = np.random.default_rng(seed)
    n, m = 1_003, 77
    return dict(encoder=np.int32(5), max_points_leaf=np.uint32(64),
                info=np.array([n, 60, 17, 77, 6], np.uint64), box=rng.random(12),
                keys=np.sort(rng.integers(0, 1 << 63, n, dtype=np.uint64)),
                perm=rng.permutation(n).astype(np.uint32), sorted_xyz=rng.random((n, 3)),
                offsets=rng.integers(0, m, m, dtype=np.uint32), ranges=rng.integers(0, n, (m, 2), dtype=np.uint64),
                centers=rng.random((m, 3)), radii=rng.random((7, 3)), half=rng.random(3),
                empty=np.zeros((0, 3), np.float64))


def _bcast_main(rank, world, port, out_path):
    import torch.distributed as dist

    from octrees_benchmark_b200.shard import broadcast_checkpoint

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = broadcast_checkpoint(_checkpoint_like(7) if rank == 1 else None, src=1)
        want = _checkpoint_like(7)
        ok = list(got) == list(want) and all(
            got[k].dtype == np.asarray(want[k]).dtype and got[k].shape == np.asarray(want[k]).shape
            and np.array_equal(got[k], want[k]) for k in want)
        ok = ok and int(got["encoder"]) == 5 and got["encoder"].ndim == 0
        with open(f"{out_path}.{rank}", "w") as f:
            f.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def test_checkpoint_broadcast_reaches_every_rank_unchanged(tmp_path):
    """One rank builds, the others restore: a checkpoint broadcast from rank 1 arrives on both ranks with
    every name, dtype, shape and byte unchanged."""
    pytest.importorskip("torch")
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "bcast")
    mp.start_processes(_bcast_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert [open(f"{out}.{r}").read() for r in range(2)] == ["ok", "ok"]
