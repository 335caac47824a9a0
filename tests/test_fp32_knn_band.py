"""The FP32 band of the group kNN filter is sound (CPU, no GPU needed).

knn_search.cu's knn_f32_threshold bounds the rounding of the FP32 squared
distance (points and query rounded once to FP32 relative to the box centre, one
FP32 difference per axis, a product and two fused adds).  This test restates
that formula and emulates the FP32 arithmetic exactly (IEEE single rounding of
each operation; a fused add as one rounding of the exact float64 value), on
tiles from 10 m to 10 km at offsets up to UTM northings, and checks that no
point at or inside a threshold is rejected."""
import math

import numpy as np
import pytest

U = 2.0 ** -24


def threshold(thr: float, ab: float) -> np.float32:
    if not thr < math.inf:
        return np.float32(np.inf)
    sr = math.sqrt(thr) * (1.0 + 1.0e-12)
    m = ab + sr
    t = sr + 1.74 * U * m
    err = 3.47 * U * m * sr + 3.01 * U * U * m * m + 3.01 * U * t * t
    value = thr + 2.0 * err
    f = np.float32(value)
    return f if float(f) >= value else np.nextafter(f, np.float32(np.inf))


def fp32_sq_distance(af: np.ndarray, bf: np.ndarray) -> np.ndarray:
    d = (af - bf).astype(np.float32)  # one FP32 rounding per axis
    x = (d[:, 0] * d[:, 0]).astype(np.float32)
    # fused multiply-add: the exact product plus the addend, rounded once (float64 holds the exact
    # product of two floats; the sum's own rounding in float64 is far below the float32 step)
    y = (d[:, 1].astype(np.float64) * d[:, 1] + x).astype(np.float32)
    return (d[:, 2].astype(np.float64) * d[:, 2] + y).astype(np.float32)


@pytest.mark.parametrize("offset", [0.0, 1.0e3, 5.0e5, 4.6e6])
@pytest.mark.parametrize("extent", [10.0, 1500.0, 10000.0])
def test_no_point_inside_the_threshold_is_rejected(offset, extent):
    rng = np.random.default_rng(int(offset) % 97 + int(extent))
    for trial in range(6):
        base = offset * rng.uniform(0.5, 1.5, 3)
        pts = base + rng.uniform(-extent / 2, extent / 2, (3000, 3))
        pts[:, 2] = base[2] + rng.uniform(-30.0, 30.0, 3000)
        c = (pts.min(0) + pts.max(0)) / 2
        radius = (pts.max(0) - pts.min(0)) / 2
        q = pts[rng.integers(0, len(pts))] + rng.normal(0.0, [0.0, 0.01, 1.0][trial % 3], 3)
        d = ((pts - q) ** 2).sum(1)
        b = q - c
        ab = (radius.max() + np.abs(b).max()) * (1.0 + 1.0e-12)
        df = fp32_sq_distance((pts - c).astype(np.float32), b.astype(np.float32))
        for thr in np.sort(d)[[0, 1, 9, 49, 199, 999, 2999]]:
            t = threshold(float(thr), ab)
            assert not np.any((d <= thr) & (df > t)), (offset, extent, trial, thr)
