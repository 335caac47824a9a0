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
