"""A replica restored from a broadcast checkpoint answers like the cloud that was built.

One rank sorts and builds, LinearOctree.checkpoint() goes through
shard.broadcast_checkpoint over NCCL (the bytes through the GPU), and
LinearOctree.from_checkpoint restores it: radius sets and kNN results must be
bitwise the built cloud's.  The process group is one rank on one GPU, in a
child process with a time bound, so that no group is left in the test process;
two-rank delivery is covered on the CPU by tests/test_shard.py."""
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import datetime, os, sys
import numpy as np
import torch
import torch.distributed as dist
from octrees_benchmark_b200 import LinearOctree
from octrees_benchmark_b200.shard import broadcast_checkpoint
from octrees_benchmark_b200.synth import lidar_tile

torch.cuda.set_device(0)
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
try:
    xyz = lidar_tile(200_000, 100.0, seed=5)
    built = LinearOctree(xyz, "hilbert", 64)
    ck = broadcast_checkpoint(built.checkpoint(), src=0)
    restored = LinearOctree.from_checkpoint(ck)
    q = xyz[::40]
    a = built.radius_search(q, 2.5, "sphere", "neighborsPrune")
    b = restored.radius_search(q, 2.5, "sphere", "neighborsPrune")
    ka, kb = built.knn(q, 20), restored.knn(q, 20)
    ok = all(np.array_equal(x, y) for x, y in zip(a, b)) and all(np.array_equal(x, y) for x, y in zip(ka, kb))
    ok = ok and int(a[0][-1]) > 0
    print("RESULT", "ok" if ok else "mismatch", flush=True)
finally:
    dist.destroy_process_group()
"""


def test_replica_from_broadcast_checkpoint_answers_like_the_built_cloud():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=180)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "RESULT ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
