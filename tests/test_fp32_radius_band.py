"""The radius search's FP32 leaf test decides only where FP64 agrees (CPU, no GPU).

radius_packet.cu's FP32 form tests a point's leaf-relative FP32 coordinates
(k_leaf_rel: each axis rounded once from the FP64 difference, w = the L1 norm
rounded up) against the query's FP32 context for that leaf (leaf_ctx) and
returns inside / outside / undecided (f32_test); undecided points take the
reference's FP64 predicate.  This test restates those three functions with an
exact emulation of their FP32 arithmetic (single rounding per operation; a
fused multiply-add as one rounding of the exact value) and checks, for sphere,
circle and cube, over leaves of many sizes and positions (offsets up to UTM
northings) and points on, near and away from the boundary, that every inside
or outside decision equals the FP64 predicate's."""
import numpy as np
import pytest

F = np.float32
S21 = F(2.0 ** -21)
S22 = F(2.0 ** -22)
FLT_MIN = F(np.finfo(np.float32).tiny)


def fma(a, b, c):
    return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)


def add_ru(a, b):
    s = np.float64(a) + np.float64(b)
    r = s.astype(np.float32)
    return np.where(r.astype(np.float64) < s, np.nextafter(r, F(np.inf)), r)


def leaf_rel(p, lc):
    v = (p - lc).astype(np.float32)
    w = add_ru(add_ru(np.abs(v[:, 0]), np.abs(v[:, 1])), np.abs(v[:, 2]))
    return v, w


def fp64_inside(kernel, p, q, r):
    if kernel == "sphere":
        d = p - q
        return ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]) < r * r
    if kernel == "circle":
        d = p - q
        return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) <= r * r
    lo, hi = q - r, q + r
    return np.all((p >= lo) & (p <= hi), axis=1)


def fp32_decide(kernel, v, w, q, r, lc):
    """1 inside, 0 outside, -1 undecided (f32_test over leaf_ctx)."""
    rf = F(r)
    if kernel in ("sphere", "circle"):
        qc = (q - lc).astype(np.float32)
        q1 = F(np.abs(qc[0]) + np.abs(qc[1]))
        if kernel == "sphere":
            q1 = F(q1 + np.abs(qc[2]))
        r2f = F(r * r)
        b0 = F(F(S21 * F(F(F(q1 + F(2.0) * rf) * rf) + r2f)) + FLT_MIN)
        b1 = F(S21 * rf)
        dx, dy = (v[:, 0] - qc[0]).astype(np.float32), (v[:, 1] - qc[1]).astype(np.float32)
        d2 = fma(dy, dy, (dx * dx).astype(np.float32))
        if kernel == "sphere":
            dz = (v[:, 2] - qc[2]).astype(np.float32)
            d2 = fma(dz, dz, d2)
        band = fma(np.full_like(w, b1), w, np.full_like(w, b0))
        out = np.full(len(v), -1)
        out[d2 < (r2f - band).astype(np.float32)] = 1
        out[d2 > (r2f + band).astype(np.float32)] = 0
        return out
    lo = ((q - r) - lc).astype(np.float32)
    hi = ((q + r) - lc).astype(np.float32)
    tlo, thi = (S22 * np.abs(lo)).astype(np.float32), (S22 * np.abs(hi)).astype(np.float32)
    tp = (S22 * w).astype(np.float32)
    out_any = np.zeros(len(v), bool)
    sure = np.ones(len(v), bool)
    for a in range(3):
        ml = (v[:, a] - lo[a]).astype(np.float32)
        mh = (hi[a] - v[:, a]).astype(np.float32)
        tl = (tp + tlo[a]).astype(np.float32)
        th = (tp + thi[a]).astype(np.float32)
        out_any |= (ml < -tl) | (mh < -th)
        sure &= (ml > tl) & (mh > th)
    return np.where(out_any, 0, np.where(sure, 1, -1))


@pytest.mark.parametrize("kernel", ["sphere", "circle", "cube"])
@pytest.mark.parametrize("offset", [0.0, 2.0e3, 4.6e6])
def test_fp32_decisions_agree_with_fp64(kernel, offset):
    rng = np.random.default_rng(int(offset) % 101 + len(kernel))
    undecided = total = 0
    for trial in range(40):
        half = rng.choice([0.05, 1.0, 20.0, 300.0])
        lc = offset * rng.uniform(0.5, 1.5, 3) + rng.uniform(-100, 100, 3)
        p = lc + rng.uniform(-half, half, (4000, 3))
        q = lc + rng.uniform(-2 * half, 2 * half, 3)
        r = float(rng.choice([0.01, 0.5, 2.5, 10.0]) * (1 + rng.uniform()))
        # points on and next to the boundary of the kernel around q
        u = rng.normal(size=(1000, 3))
        u /= np.linalg.norm(u, axis=1)[:, None]
        if kernel == "cube":
            u = np.sign(u) * (np.abs(u) == np.abs(u).max(1)[:, None])
        shell = q + u * r * (1 + rng.choice([-1e-12, 0.0, 1e-12, 1e-7, -1e-7], (1000, 1)))
        p = np.concatenate([p, shell])
        v, w = leaf_rel(p, lc)
        exact = fp64_inside(kernel, p, q, r)
        dec = fp32_decide(kernel, v, w, q, r, lc)
        assert not np.any((dec == 1) & ~exact), (kernel, offset, trial)
        assert not np.any((dec == 0) & exact), (kernel, offset, trial)
        undecided += int((dec == -1).sum())
        total += len(p)
    assert undecided < total  # the filter decides most points
