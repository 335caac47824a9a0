"""Generate the golden fixtures from the UNMODIFIED reference implementation.

    make -C oracle ref && python tests/golden/make_golden.py

Runs the reference (compiled from its own headers by oracle/Makefile, bridged by
oracle/ref_bridge.cpp) on small seeded clouds and writes what it returns:
sorted keys, point ids, the Box, the octree arrays, radius-search results for
every kernel and variant, neighborsStruct ranges and kNN results, plus tables
of anchor coordinates (including the flat-axis and out-of-range edge cases)
and of Morton / Hilbert keys.  The fixtures are committed, so the tests do
not need the reference sources; this script does.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from octrees_benchmark_b200.synth import lidar_tile, query_indices  # noqa: E402
from oracle.oracle import Reference, build_reference  # noqa: E402

RADII = {"sphere": 1, "circle": 0, "cube": 3, "square": 2}


def csr_sorted(offs, idx):
    out = np.empty_like(idx)
    for q in range(len(offs) - 1):
        a, b = int(offs[q]), int(offs[q + 1])
        out[a:b] = np.sort(idx[a:b])
    return out


def cloud_fixture(name, xyz, encoder, leaf, radii, ks, n_queries=40, extra_centers=None):
    R = Reference(encoder, xyz, leaf, threads=1)
    sxyz, ids, keys = R.points()
    arr = R.arrays()
    q = sxyz[query_indices(n_queries, len(sxyz), seed=7)] if len(sxyz) else np.zeros((0, 3))
    if extra_centers is not None:
        q = np.concatenate([q, extra_centers])
    out = dict(xyz=xyz, encoder=encoder, max_leaf=leaf, keys=keys, ids=ids, sorted_xyz=sxyz, box=R.box(),
               info=np.array([R.n, R.n_leaf, R.n_internal, R.n_total, R.max_depth], np.uint64), centers=q,
               radii=np.array(radii, np.float64), ks=np.array(ks, np.int64), **{"tree_" + k: v for k, v in arr.items()})
    for ri, r in enumerate(radii):
        for kn, kv in RADII.items():
            for algo in (1, 2, 3):
                offs, idx = R.radius(kv, algo, q, r, threads=1)
                out[f"rad_{ri}_{kn}_{algo}_offs"] = offs
                out[f"rad_{ri}_{kn}_{algo}_idx"] = csr_sorted(offs, idx)
            offs, pairs = R.struct_ranges(kv, q, r, threads=1)
            order = []
            for qq in range(len(offs) - 1):
                a, b = int(offs[qq]), int(offs[qq + 1])
                seg = pairs[a:b]
                order.append(seg[np.lexsort((seg[:, 1], seg[:, 0]))] if len(seg) else seg)
            out[f"struct_{ri}_{kn}_offs"] = offs
            out[f"struct_{ri}_{kn}_pairs"] = np.concatenate(order) if order else pairs
    for k in ks:
        idx, d2, cnt = R.knn(q, k, threads=1)
        out[f"knn_{k}_idx"] = idx
        out[f"knn_{k}_d2"] = d2
        out[f"knn_{k}_cnt"] = cnt
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "n", len(xyz), "nodes", R.n_total, "depth", R.max_depth)


def main():
    if build_reference() is None:
        raise SystemExit("the reference sources are needed to regenerate the fixtures")
    # synthetic LiDAR tiles (terrain + cylinders), both encoders
    cloud_fixture("tile_morton_leaf16", lidar_tile(2500, 25.0, seed=11), 1, 16, [0.7, 2.0], [1, 7, 16])
    cloud_fixture("tile_hilbert_leaf32", lidar_tile(3000, 27.0, seed=12), 5, 32, [1.0, 3.0], [1, 10, 33])
    # degenerate plane z = 0 (flat axis: radius 0, anchor coordinate NaN -> max)
    g = np.stack(np.meshgrid(np.arange(20) * 0.1, np.arange(20) * 0.1, indexing="ij"), -1).reshape(-1, 2)
    plane = np.concatenate([g, np.zeros((len(g), 1))], 1)
    cloud_fixture("plane_morton_leaf8", plane, 1, 8, [0.15, 0.5], [1, 4, 9])
    # degenerate line along x with duplicates and a 1e6 offset
    line = np.stack([1e6 + np.repeat(np.arange(60) * 0.1, 2), np.full(120, 1e6), np.full(120, 1e6)], 1)
    cloud_fixture("line_hilbert_leaf4", line, 5, 4, [0.0, 0.35], [1, 3, 8],
                  extra_centers=np.array([[1e6 + 2.05, 1e6, 1e6], [1e6 - 5, 1e6, 1e6]]))
    # anchor coordinates incl. edge cases (flat axis, outside the box, NaN, inf)
    rng = np.random.default_rng(5)
    pcr = [(0.0, 0.0, 0.0), (1.0, 1.0, 0.0), (0.5, 0.0, 1.0), (-1.0, 0.0, 1.0), (1.0, 0.0, 1.0),
           (-1.0000001, 0.0, 1.0), (-1.5, 0.0, 1.0), (-3.0, 0.0, 1.0), (5.0, 0.0, 1.0), (np.nan, 0.0, 1.0),
           (np.inf, 0.0, 1.0), (-np.inf, 0.0, 1.0), (1e300, 0.0, 1e-300)]
    for _ in range(200):
        c = rng.uniform(-1e3, 1e3)
        r = rng.uniform(1e-3, 1e3)
        pcr.append((rng.uniform(c - r, c + r), c, r))
    pcr = np.array(pcr, np.float64)
    anchors = np.array([Reference.anchor(*t) for t in pcr], np.uint64)
    coords = rng.integers(0, 1 << 21, (500, 3), dtype=np.uint64)
    coords[:4] = [[0, 0, 0], [(1 << 21) - 1] * 3, [1000, 2000, 3000], [1, 0, 0]]
    mk = np.array([Reference.encode_xyz(1, *map(int, c)) for c in coords], np.uint64)
    hk = np.array([Reference.encode_xyz(5, *map(int, c)) for c in coords], np.uint64)
    md = np.array([Reference.decode_key(1, int(k)) for k in mk], np.uint64)
    hd = np.array([Reference.decode_key(5, int(k)) for k in hk], np.uint64)
    np.savez_compressed(os.path.join(HERE, "keys_anchor.npz"), pcr=pcr, anchors=anchors, coords=coords,
                        morton=mk, hilbert=hk, morton_dec=md, hilbert_dec=hd)
    print("keys_anchor", len(pcr), len(coords))


if __name__ == "__main__":
    main()
