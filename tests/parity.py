"""Parity helpers shared by the tests: exact comparisons of keys, trees,
neighbour sets and kNN results.

The bar is bit-exactness: keys, permutations, tree arrays and every radius
neighbour set (compared as sorted index sets) must be identical; kNN squared
distances must be bitwise identical, index sets identical below the k-th
distance, and at the k-th distance the device must hold the lowest indices of
all points at exactly that distance (the reference's heap leaves the order of
equal distances unspecified, linear_octree.hpp:837-840).
"""
from __future__ import annotations

import numpy as np


def same_f64(a, b) -> bool:
    """Bitwise equality of float64 arrays, treating every NaN as equal."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.shape != b.shape:
        return False
    an, bn = np.isnan(a), np.isnan(b)
    if not np.array_equal(an, bn):
        return False
    return np.array_equal(a[~an].view(np.uint64), b[~bn].view(np.uint64))


def sorted_csr(offs, idx):
    offs = np.asarray(offs, np.int64)
    idx = np.asarray(idx, np.int64)
    out = idx.copy()
    for q in range(len(offs) - 1):
        a, b = offs[q], offs[q + 1]
        out[a:b] = np.sort(idx[a:b])
    return out


def assert_csr_equal(offs_a, idx_a, offs_b, idx_b, what=""):
    offs_a = np.asarray(offs_a, np.int64)
    offs_b = np.asarray(offs_b, np.int64)
    if not np.array_equal(offs_a, offs_b):
        cnt_a, cnt_b = np.diff(offs_a), np.diff(offs_b)
        bad = np.nonzero(cnt_a != cnt_b)[0]
        raise AssertionError(f"{what}: counts differ on {len(bad)} queries, first {bad[:5]} "
                             f"({cnt_a[bad[:5]]} vs {cnt_b[bad[:5]]})")
    a = sorted_csr(offs_a, idx_a)
    b = sorted_csr(offs_b, idx_b)
    if not np.array_equal(a, b):
        pos = np.nonzero(a != b)[0][0]
        q = int(np.searchsorted(offs_a, pos, side="right") - 1)
        raise AssertionError(f"{what}: neighbour sets differ, first at query {q}")


def assert_ranges_equal(offs_a, pairs_a, offs_b, pairs_b, what=""):
    """neighborsStruct ranges compared as per-query sorted lists of (first, last)."""
    offs_a = np.asarray(offs_a, np.int64)
    offs_b = np.asarray(offs_b, np.int64)
    assert np.array_equal(offs_a, offs_b), f"{what}: range counts differ"
    pa = np.asarray(pairs_a, np.int64).reshape(-1, 2)
    pb = np.asarray(pairs_b, np.int64).reshape(-1, 2)
    for q in range(len(offs_a) - 1):
        a, b = offs_a[q], offs_a[q + 1]
        sa = pa[a:b][np.lexsort((pa[a:b, 1], pa[a:b, 0]))]
        sb = pb[a:b][np.lexsort((pb[a:b, 1], pb[a:b, 0]))]
        assert np.array_equal(sa, sb), f"{what}: ranges differ at query {q}"


def sq_dist(xyz, c):
    """distPointsSquared(center, point) in the reference's operation order."""
    dx = c[0] - xyz[:, 0]
    dy = c[1] - xyz[:, 1]
    dz = c[2] - xyz[:, 2]
    return dx * dx + dy * dy + dz * dz


def assert_knn_equal(idx_g, d2_g, cnt_g, idx_r, d2_r, cnt_r, xyz, centers, what="", lowest_ties=True):
    """kNN result g (ascending by distance) against r (the reference or the oracle).

    Squared distances bitwise equal, index sets equal below the k-th distance.
    At the k-th distance, with ``lowest_ties`` g must hold the lowest indices
    of all points at exactly that distance (the device's and the oracle's
    rule); without it any such points are accepted (the reference's heap order
    of equal distances is unspecified)."""
    idx_g = np.asarray(idx_g, np.int64)
    idx_r = np.asarray(idx_r, np.int64)
    cnt_g = np.asarray(cnt_g, np.int64)
    cnt_r = np.asarray(cnt_r, np.int64)
    assert np.array_equal(cnt_g, cnt_r), f"{what}: counts differ"
    n_ties = 0
    for q in range(len(cnt_g)):
        c = int(cnt_g[q])
        if c == 0:
            continue
        dg, dr = d2_g[q, :c], d2_r[q, :c]
        assert same_f64(dg, dr), f"{what}: squared distances differ at query {q}"
        kth = dg[c - 1]
        below_g = np.sort(idx_g[q, :c][dg < kth])
        below_r = np.sort(idx_r[q, :c][dr < kth])
        assert np.array_equal(below_g, below_r), f"{what}: index sets below the k-th distance differ at query {q}"
        tie_g = idx_g[q, :c][dg == kth]
        tie_r = idx_r[q, :c][dr == kth]
        if np.array_equal(np.sort(tie_g), np.sort(tie_r)):
            continue
        n_ties += 1
        allk = np.nonzero(sq_dist(xyz, centers[q]) == kth)[0]
        if lowest_ties:
            want = np.sort(allk)[: len(tie_g)]
            assert np.array_equal(np.sort(tie_g), want), f"{what}: tie group at query {q} is not the lowest indices"
        else:
            assert len(tie_g) == len(tie_r) and np.all(np.isin(tie_g, allk)), f"{what}: bad tie group at query {q}"
    return n_ties


# ---- vectorised counts of differences (large query sets) --------------------
def csr_set_diffs(offs_a, idx_a, offs_b, idx_b) -> int:
    """Number of queries whose neighbour sets differ between two CSR results
    (the order within a query is free)."""
    offs_a = np.asarray(offs_a, np.int64)
    offs_b = np.asarray(offs_b, np.int64)
    idx_a = np.asarray(idx_a, np.int64)[: offs_a[-1]]
    idx_b = np.asarray(idx_b, np.int64)[: offs_b[-1]]
    ca, cb = np.diff(offs_a), np.diff(offs_b)
    nq = len(ca)
    same_cnt = ca == cb
    bad = ~same_cnt
    keep_a = np.repeat(same_cnt, ca)
    keep_b = np.repeat(same_cnt, cb)
    seg = np.repeat(np.arange(nq), np.where(same_cnt, ca, 0))
    va, vb = idx_a[keep_a], idx_b[keep_b]
    sa = va[np.lexsort((va, seg))]
    sb = vb[np.lexsort((vb, seg))]
    diff = sa != sb
    if diff.any():
        bad[np.unique(seg[diff])] = True
    return int(bad.sum())


def knn_diffs(idx_g, d2_g, cnt_g, idx_r, d2_r, cnt_r, xyz, centers, max_tie_checks: int = 64):
    """kNN result g against reference r, vectorised.  Returns (queries that
    differ, max |d2_g - d2_r|, tie groups checked by brute force).  A query
    differs when its count, any squared distance (bitwise) or its index set
    below the k-th distance differs, or when its tie group at the k-th
    distance is not the lowest indices of all points at that distance."""
    idx_g = np.asarray(idx_g, np.int64)
    idx_r = np.asarray(idx_r, np.int64)
    d2_g = np.asarray(d2_g, np.float64)
    d2_r = np.asarray(d2_r, np.float64)
    cnt_g = np.asarray(cnt_g, np.int64)
    cnt_r = np.asarray(cnt_r, np.int64)
    nq, k = d2_g.shape
    bad = cnt_g != cnt_r
    valid = np.arange(k)[None, :] < np.minimum(cnt_g, cnt_r)[:, None]
    err = np.where(valid, np.abs(d2_g - d2_r), 0.0)
    max_err = float(err.max()) if err.size else 0.0
    bad |= ((d2_g.view(np.uint64) != d2_r.view(np.uint64)) & valid).any(axis=1)
    last = np.maximum(np.minimum(cnt_g, cnt_r) - 1, 0)
    kth = d2_g[np.arange(nq), last][:, None]
    big = np.iinfo(np.int64).max
    below_g = np.sort(np.where(valid & (d2_g < kth), idx_g, big), axis=1)
    below_r = np.sort(np.where(valid & (d2_r < kth), idx_r, big), axis=1)
    bad |= (below_g != below_r).any(axis=1)
    tie_g = np.sort(np.where(valid & (d2_g == kth), idx_g, big), axis=1)
    tie_r = np.sort(np.where(valid & (d2_r == kth), idx_r, big), axis=1)
    tie_rows = np.nonzero(~bad & (tie_g != tie_r).any(axis=1))[0]
    checked = 0
    for q in tie_rows[:max_tie_checks]:
        checked += 1
        allk = np.sort(np.nonzero(sq_dist(xyz, centers[q]) == kth[q, 0])[0])
        mine = tie_g[q][tie_g[q] != big]
        if not np.array_equal(mine, allk[: len(mine)]):
            bad[q] = True
    bad[tie_rows[max_tie_checks:]] = True  # not checked: counted as differences
    return int(bad.sum()), max_err, checked


def ranges_diffs(offs_a, pairs_a, offs_b, pairs_b) -> int:
    """Number of queries whose neighborsStruct ranges differ, each query's
    ranges compared as a sorted list of (first, last) pairs."""
    offs_a = np.asarray(offs_a, np.int64)
    offs_b = np.asarray(offs_b, np.int64)
    pa = np.asarray(pairs_a, np.int64).reshape(-1, 2)[: offs_a[-1]]
    pb = np.asarray(pairs_b, np.int64).reshape(-1, 2)[: offs_b[-1]]
    ca, cb = np.diff(offs_a), np.diff(offs_b)
    same = ca == cb
    bad = ~same
    seg = np.repeat(np.arange(len(ca)), np.where(same, ca, 0))
    va, vb = pa[np.repeat(same, ca)], pb[np.repeat(same, cb)]
    sa = va[np.lexsort((va[:, 1], va[:, 0], seg))]
    sb = vb[np.lexsort((vb[:, 1], vb[:, 0], seg))]
    diff = (sa != sb).any(axis=1)
    if diff.any():
        bad[np.unique(seg[diff])] = True
    return int(bad.sum())


MIX64_C = (0x9E3779B97F4A7C15, 0xBF58476D1CE4E5B9, 0x94D049BB133111EB)


def mix64_np(v):
    """splitmix64's output function on uint64 values (the set-hash term of the
    reference bridge's refo_radius_hash)."""
    z = np.asarray(v, np.uint64) + np.uint64(MIX64_C[0])
    z = (z ^ (z >> np.uint64(30))) * np.uint64(MIX64_C[1])
    z = (z ^ (z >> np.uint64(27))) * np.uint64(MIX64_C[2])
    return z ^ (z >> np.uint64(31))


def mix64_torch(t):
    """mix64_np on an int64 torch tensor (two's complement wrap-around, logical
    right shifts by masking)."""
    def s64(c):
        return c - (1 << 64) if c >= (1 << 63) else c

    def srl(z, s):
        return (z >> s) & ((1 << (64 - s)) - 1)

    import torch

    z = t.to(torch.int64) + s64(MIX64_C[0])
    z = (z ^ srl(z, 30)) * s64(MIX64_C[1])
    z = (z ^ srl(z, 27)) * s64(MIX64_C[2])
    return z ^ srl(z, 31)


def csr_count_hash_torch(offs, idx):
    """Per-query (count, sum of mix64(index) mod 2^64) of a device CSR result,
    as int64 tensors (the hash's bits are those of the uint64 sum)."""
    import torch

    offs = offs.to(torch.int64)
    h = mix64_torch(idx[: int(offs[-1].item())].to(torch.int64))
    cs = torch.cat([torch.zeros(1, dtype=torch.int64, device=h.device), torch.cumsum(h, 0)])
    return offs[1:] - offs[:-1], cs[offs[1:]] - cs[offs[:-1]]
