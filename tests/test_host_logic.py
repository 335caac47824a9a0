"""Host-side logic that needs no GPU: the Hilbert state table compiled into the
kernels, the synthetic generator's determinism, and the header parser."""
import os
import re

import numpy as np

from octrees_benchmark_b200 import capi
from octrees_benchmark_b200.synth import batched_clouds, config_cloud, lidar_tile, query_indices

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _gen_table():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen_hilbert_table", os.path.join(ROOT, "octrees_benchmark_b200", "csrc", "gen_hilbert_table.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.table()


def _table_encode(rows, x, y, z):
    s, k = 0, 0
    for level in range(20, -1, -1):
        o = (((x >> level) & 1) << 2) | (((y >> level) & 1) << 1) | ((z >> level) & 1)
        e = rows[s][o]
        k = (k << 3) | (e & 7)
        s = e >> 3
    return k


def test_hilbert_table_reproduces_reference_keys(port):
    rows = _gen_table()
    assert len(rows) == 24 and all(len(r) == 8 for r in rows)
    rng = np.random.default_rng(9)
    coords = rng.integers(0, 1 << 21, (3000, 3))
    coords[:3] = [[0, 0, 0], [(1 << 21) - 1] * 3, [1000, 2000, 3000]]
    for x, y, z in coords:
        assert _table_encode(rows, int(x), int(y), int(z)) == port.encode_xyz(5, int(x), int(y), int(z))


def test_hilbert_table_in_kernel_source_is_the_generated_one():
    src = open(os.path.join(ROOT, "octrees_benchmark_b200", "csrc", "sfc.cuh")).read()
    body = re.search(r"kHilbertTable\[kHilbertStates \* 8\] = \{(.*?)\};", src, re.S).group(1)
    vals = [int(v) for v in re.findall(r"\d+", body)]
    assert vals == [v for row in _gen_table() for v in row]


def test_synthetic_generator_is_deterministic():
    a = lidar_tile(5000, 60.0, seed=3)
    b = lidar_tile(5000, 60.0, seed=3)
    assert np.array_equal(a, b) and a.shape == (5000, 3) and a.dtype == np.float64
    assert not np.array_equal(a, lidar_tile(5000, 60.0, seed=4))
    assert a[:, 0].min() >= 0 and a[:, 0].max() <= 60.0
    xyz, cfg = config_cloud("c2_10M_hilbert", n=20000)
    assert cfg["n"] == 20000 and cfg["encoder"] == 5 and cfg["max_leaf"] == 64 and xyz.shape == (20000, 3)
    q = query_indices(100, 5000)
    assert q.min() >= 0 and q.max() < 5000 and np.array_equal(q, query_indices(100, 5000))
    clouds = batched_clouds(16)
    assert len(clouds) == 16 and all(10_000 <= c["n"] <= 2_000_000 for c in clouds)
    assert {c["max_leaf"] for c in batched_clouds(256)} <= {32, 64, 128}


def test_header_parser_lists_every_entry_point():
    names = capi.header_functions()
    for must in ("oct_cloud_create", "oct_encode_sort", "oct_build", "oct_radius_search", "oct_struct_search",
                 "oct_knn", "oct_encode_sort_noalloc", "oct_set_search_config"):
        assert must in names
