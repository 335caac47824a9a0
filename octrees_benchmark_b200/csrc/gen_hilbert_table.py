"""Generate the 24-state Hilbert table used by csrc/sfc.cuh.

The reference's HilbertEncoder3D::encode (inc/encoding/hilbert_encoder_3d.hpp:29-66)
walks 21 levels; at each level it maps the current octant through
{0,1,3,2,7,6,4,5}, inverts some of the (transformed) coordinates and rotates or
swaps them.  After any number of levels the transformed coordinates are the
original ones under an axis permutation and per-axis inversion, so the encoder
is a finite automaton over (permutation, inversions) states.  This script
follows the reference's per-level rules on that state, keeps the states
reachable from the identity (24 of the 48), and prints the table rows:
entry = next_state << 3 | digit, indexed [state][octant of the original
coordinates (x << 2 | y << 1 | z)].  Run: python gen_hilbert_table.py
"""
import itertools

LUT = [0, 1, 3, 2, 7, 6, 4, 5]


def step(perm, flips, bits):
    f = [(flips >> 2) & 1, (flips >> 1) & 1, flips & 1]
    xi, yi, zi = (bits[perm[a]] ^ f[a] for a in range(3))
    digit = LUT[(xi << 2) | (yi << 1) | zi]
    nyi, nzi = 1 - yi, 1 - zi
    f = [f[0] ^ (xi & (nyi | zi)), f[1] ^ ((xi & (yi | zi)) | (yi & nzi)), f[2] ^ ((xi & nyi & nzi) | (yi & nzi))]
    p = list(perm)
    if zi:                      # x, y, z <- y, z, x
        p, f = [p[1], p[2], p[0]], [f[1], f[2], f[0]]
    elif not yi:                # swap x and z
        p, f = [p[2], p[1], p[0]], [f[2], f[1], f[0]]
    return digit, (tuple(p), (f[0] << 2) | (f[1] << 1) | f[2])


def table():
    init = ((0, 1, 2), 0)
    states, frontier = [init], [init]
    while frontier:
        s = frontier.pop()
        for o in range(8):
            _, n = step(*s, ((o >> 2) & 1, (o >> 1) & 1, o & 1))
            if n not in states:
                states.append(n)
                frontier.append(n)
    ordered = [init] + sorted(s for s in states if s != init)
    index = {s: i for i, s in enumerate(ordered)}
    rows = []
    for s in ordered:
        row = []
        for o in range(8):
            d, n = step(*s, ((o >> 2) & 1, (o >> 1) & 1, o & 1))
            row.append((index[n] << 3) | d)
        rows.append(row)
    return rows


if __name__ == "__main__":
    for row in table():
        print("    " + ", ".join(f"{v:3d}" for v in row) + ",")
