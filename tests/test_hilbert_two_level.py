"""k_encode's two-level Hilbert walk gives the reference's keys (CPU, no GPU).

sfc.cuh composes its 24-state automaton table (state, octant -> next state,
digit) with itself into a 24 x 64 table (hilbert_table2_fill) and walks 21
levels as one single step then ten two-level steps, reading the octant pairs
from one bit interleave with x in the high bit of each triple
(hilbert_encode_tbl2).  This test reads the one-level table from the source,
restates the composition and the walk, and checks the keys against the
one-level walk and against the oracle's Hilbert encoder (the reference's
21-level loop) on random and corner coordinates."""
import os
import re

import numpy as np

from oracle.oracle import Port

SFC = os.path.join(os.path.dirname(__file__), "..", "octrees_benchmark_b200", "csrc", "sfc.cuh")


def table():
    src = open(SFC).read()
    body = src[src.index("kHilbertTable[kHilbertStates * 8] = {"):]
    body = body[body.index("{") + 1:body.index("};")]
    t = [int(v) for v in re.findall(r"\d+", body)]
    assert len(t) == 24 * 8
    return t


def spread3(v):
    r = 0
    for i in range(21):
        r |= ((v >> i) & 1) << (3 * i)
    return r


def walk1(t, x, y, z):
    key, st = 0, 0
    for level in range(20, -1, -1):
        o = (((x >> level) & 1) << 2) | (((y >> level) & 1) << 1) | ((z >> level) & 1)
        e = t[st * 8 + o]
        key = (key << 3) | (e & 7)
        st = e >> 3
    return key


def table2(t):
    t2 = []
    for i in range(24 * 64):
        e1 = t[(i >> 6) * 8 + ((i >> 3) & 7)]
        e2 = t[(e1 >> 3) * 8 + (i & 7)]
        t2.append(((e2 >> 3) << 6) | ((e1 & 7) << 3) | (e2 & 7))
    return t2


def walk2(t, t2, x, y, z):
    m = spread3(z) | (spread3(y) << 1) | (spread3(x) << 2)
    e = t[(m >> 60) & 7]
    key, st = e & 7, e >> 3
    for level in range(19, 0, -2):
        e2 = t2[st * 64 + ((m >> (3 * (level - 1))) & 63)]
        key = (key << 6) | (e2 & 63)
        st = e2 >> 6
    return key


def test_two_level_walk_equals_reference_keys():
    t = table()
    t2 = table2(t)
    assert max(t2) < 1 << 16  # fits the kernel's uint16 entries
    port = Port()
    rng = np.random.default_rng(11)
    top = (1 << 21) - 1
    coords = [(0, 0, 0), (top, top, top), (top, 0, 0), (0, top, 0), (0, 0, top), (1 << 20, 1 << 20, 1 << 20)]
    coords += [tuple(int(v) for v in rng.integers(0, 1 << 21, 3)) for _ in range(3000)]
    for x, y, z in coords:
        k2 = walk2(t, t2, x, y, z)
        assert k2 == walk1(t, x, y, z)
        assert k2 == port.encode_xyz(5, x, y, z)
