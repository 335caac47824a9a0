"""Deterministic synthetic airborne-LiDAR tiles.

The reference benchmarks real clouds (Paris-Lille-3D, DALES, Semantic3D,
Speulderbos; bench_neighbors.bash:7-21) that are not available here; these
seeded tiles stand in for them with the same shape of data:

* x, y uniform over a square tile of side ``tile_m`` metres;
* 85 % of the points are terrain: z = sum of 4 sinusoids (wavelengths 50, 100,
  200 and 400 m, random directions and phases, total amplitude 20 m) plus
  Gaussian noise of sigma 0.05 m;
* 15 % are canopy/building clusters: ``n_cyl`` vertical cylinders of radius
  2-15 m; points are area-uniform in the cylinder's disk, with z uniform from
  the terrain up to the cylinder's height (3-25 m above the terrain).

Everything is drawn from ``numpy.random.default_rng(seed)``, so a (n, tile,
seed) triple always gives the same float64 (n, 3) array.  Query centres are
cloud points picked uniformly at random: ``search_set`` reproduces the
reference's SearchSet (inc/benchmarking/search_set.hpp:23-44) index for index
(mt19937 seeded 42, uniform_int_distribution); ``query_indices`` draws other
seeded sets from numpy's PCG64.
"""
from __future__ import annotations

import math

import numpy as np

WAVELENGTHS = (50.0, 100.0, 200.0, 400.0)
AMPLITUDE = 20.0 / len(WAVELENGTHS)


def _terrain(x, y, dirs, phases):
    z = np.zeros_like(x)
    for lam, th, ph in zip(WAVELENGTHS, dirs, phases):
        z += AMPLITUDE * np.sin((2.0 * math.pi / lam) * (x * math.cos(th) + y * math.sin(th)) + ph)
    return z


def lidar_tile(n: int, tile_m: float, seed: int, n_cyl: int = 300, canopy_frac: float = 0.15,
               noise: float = 0.05) -> np.ndarray:
    """One synthetic tile of ``n`` points, float64 (n, 3), in random order."""
    rng = np.random.default_rng(seed)
    dirs = rng.uniform(0.0, math.pi, len(WAVELENGTHS))
    phases = rng.uniform(0.0, 2.0 * math.pi, len(WAVELENGTHS))
    n_can = int(round(n * canopy_frac)) if n_cyl > 0 else 0
    n_ter = n - n_can
    out = np.empty((n, 3), np.float64)
    x = rng.uniform(0.0, tile_m, n_ter)
    y = rng.uniform(0.0, tile_m, n_ter)
    out[:n_ter, 0] = x
    out[:n_ter, 1] = y
    out[:n_ter, 2] = _terrain(x, y, dirs, phases) + rng.normal(0.0, noise, n_ter)
    if n_can:
        cr = np.minimum(rng.uniform(2.0, 15.0, n_cyl), 0.25 * tile_m)
        cx = rng.uniform(cr, tile_m - cr)
        cy = rng.uniform(cr, tile_m - cr)
        ch = rng.uniform(3.0, 25.0, n_cyl)
        w = cr * cr
        which = rng.choice(n_cyl, size=n_can, p=w / w.sum())
        rad = cr[which] * np.sqrt(rng.uniform(0.0, 1.0, n_can))
        ang = rng.uniform(0.0, 2.0 * math.pi, n_can)
        px = cx[which] + rad * np.cos(ang)
        py = cy[which] + rad * np.sin(ang)
        out[n_ter:, 0] = px
        out[n_ter:, 1] = py
        out[n_ter:, 2] = _terrain(px, py, dirs, phases) + rng.uniform(0.0, 1.0, n_can) * ch[which]
    # random input order, as a LAS file would deliver it
    return out[rng.permutation(n)]


def large_tile_device(n: int = 500_000_000, tile_m: float = 10_000.0, seed: int = 3, urban_frac: float = 0.4,
                      n_clusters: int = 50, rural_density: float = 5.0, chunk: int = 50_000_000):
    """A large skewed tile generated on the current CUDA device (torch, float64 (n, 3)).

    Rural ground: ``(1 - urban_frac) n`` points at ``rural_density`` points/m^2
    over a full-width band of the tile (its depth follows from the density),
    z = the terrain of ``lidar_tile`` + N(0, 0.05 m).  Urban: ``urban_frac n``
    points in ``n_clusters`` building clusters of radius 10-40 m anywhere on
    the tile, each cluster's share proportional to its footprint (with the
    defaults about 1,800-2,000 points/m^2), z uniform from the terrain up to the
    building's height (5-30 m).  Drawn from a seeded CUDA generator in chunks;
    rural points come first, then urban (the pipeline sorts them anyway)."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(seed)
    dirs = rng.uniform(0.0, math.pi, len(WAVELENGTHS))
    phases = rng.uniform(0.0, 2.0 * math.pi, len(WAVELENGTHS))

    def terrain(x, y):
        z = torch.zeros_like(x)
        for lam, th, ph in zip(WAVELENGTHS, dirs, phases):
            z += AMPLITUDE * torch.sin((2.0 * math.pi / lam) * (x * math.cos(th) + y * math.sin(th)) + ph)
        return z

    out = torch.empty((n, 3), dtype=torch.float64, device=dev)
    n_urb = int(round(n * urban_frac))
    n_rur = n - n_urb
    depth = min(tile_m, n_rur / (rural_density * tile_m)) if n_rur else 0.0
    for s in range(0, n_rur, chunk):
        m = min(chunk, n_rur - s)
        x = torch.rand(m, dtype=torch.float64, device=dev, generator=g) * tile_m
        y = torch.rand(m, dtype=torch.float64, device=dev, generator=g) * depth
        out[s:s + m, 0] = x
        out[s:s + m, 1] = y
        out[s:s + m, 2] = terrain(x, y) + 0.05 * torch.randn(m, dtype=torch.float64, device=dev, generator=g)
    if n_urb:
        cr = torch.tensor(rng.uniform(10.0, 40.0, n_clusters), dtype=torch.float64, device=dev)
        cx = torch.tensor(rng.uniform(40.0, tile_m - 40.0, n_clusters), dtype=torch.float64, device=dev)
        cy = torch.tensor(rng.uniform(40.0, tile_m - 40.0, n_clusters), dtype=torch.float64, device=dev)
        ch = torch.tensor(rng.uniform(5.0, 30.0, n_clusters), dtype=torch.float64, device=dev)
        w = cr * cr
        for s in range(0, n_urb, chunk):
            m = min(chunk, n_urb - s)
            which = torch.multinomial(w, m, replacement=True, generator=g)
            rad = cr[which] * torch.sqrt(torch.rand(m, dtype=torch.float64, device=dev, generator=g))
            ang = torch.rand(m, dtype=torch.float64, device=dev, generator=g) * (2.0 * math.pi)
            px = cx[which] + rad * torch.cos(ang)
            py = cy[which] + rad * torch.sin(ang)
            o = n_rur + s
            out[o:o + m, 0] = px
            out[o:o + m, 1] = py
            out[o:o + m, 2] = terrain(px, py) + torch.rand(m, dtype=torch.float64, device=dev, generator=g) * ch[which]
    return out


def query_indices(n_queries: int, cloud_size: int, seed: int = 42) -> np.ndarray:
    """Random centre indices into the (sorted) cloud from numpy's PCG64 (seeded sets for the tests and the
    bench's per-step batches); ``search_set`` gives the reference's own SearchSet stream."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, cloud_size, n_queries, dtype=np.int64)


class MT19937:
    """The 32-bit Mersenne Twister of Matsumoto and Nishimura (1998), as
    std::mt19937: seeded by the init_genrand recurrence, 624-word twist,
    tempered 32-bit outputs.  The twist is vectorised in the three blocks
    whose inputs are already final (i < 227 reads only old words; 227 <= i <
    454 and 454 <= i < 623 read words the previous block rewrote; i = 623 reads
    the new word 0)."""

    N, M = 624, 397
    MATRIX_A, UPPER, LOWER = 0x9908B0DF, 0x80000000, 0x7FFFFFFF

    def __init__(self, seed: int = 5489):
        mt = [int(seed) & 0xFFFFFFFF]
        for i in range(1, self.N):
            prev = mt[-1]
            mt.append((1812433253 * (prev ^ (prev >> 30)) + i) & 0xFFFFFFFF)
        self.mt = np.array(mt, np.uint64)
        self.pos = self.N

    def _twist_block(self, lo, hi, nxt, far):
        y = (self.mt[lo:hi] & self.UPPER) | (nxt & self.LOWER)
        self.mt[lo:hi] = far ^ (y >> np.uint64(1)) ^ np.where((y & np.uint64(1)) != 0, np.uint64(self.MATRIX_A),
                                                              np.uint64(0))

    def _twist(self):
        mt, N, M = self.mt, self.N, self.M
        self._twist_block(0, N - M, mt[1:N - M + 1].copy(), mt[M:N].copy())
        self._twist_block(N - M, 2 * (N - M), mt[N - M + 1:2 * (N - M) + 1].copy(), mt[0:N - M].copy())
        self._twist_block(2 * (N - M), N - 1, mt[2 * (N - M) + 1:N].copy(), mt[N - M:M - 1].copy())
        self._twist_block(N - 1, N, mt[0:1].copy(), mt[M - 1:M].copy())
        self.pos = 0

    @staticmethod
    def _temper(y):
        y = y.copy()
        y ^= y >> np.uint64(11)
        y ^= (y << np.uint64(7)) & np.uint64(0x9D2C5680)
        y ^= (y << np.uint64(15)) & np.uint64(0xEFC60000)
        y ^= y >> np.uint64(18)
        return y & np.uint64(0xFFFFFFFF)

    def _peek(self, n: int) -> np.ndarray:
        """Up to n next outputs from the current state block, without consuming them."""
        if self.pos >= self.N:
            self._twist()
        return self._temper(self.mt[self.pos:self.pos + min(n, self.N - self.pos)])

    def next_u32(self, n: int) -> np.ndarray:
        out = []
        while n > 0:
            y = self._peek(n)
            self.pos += len(y)
            n -= len(y)
            out.append(y)
        return np.concatenate(out) if out else np.empty(0, np.uint64)

    def uniform_int(self, n: int, lo: int, hi: int) -> np.ndarray:
        """n draws of std::uniform_int_distribution(lo, hi) with a 32-bit engine and a range below 2^32:
        Lemire's nearly divisionless method (2019) - the 64-bit product of a draw and the range, its high
        word the value, a draw rejected while its low word is below 2^32 mod range."""
        rng = hi - lo + 1
        assert 0 < rng < (1 << 32)
        thresh = np.uint64(((1 << 32) - rng) % rng)
        parts, got = [], 0
        while got < n:
            x = self._peek(n - got)
            prod = x * np.uint64(rng)
            ok = (prod & np.uint64(0xFFFFFFFF)) >= thresh
            take = len(x) if ok.all() else int(np.argmin(ok))  # accepted draws before the first rejection
            parts.append(prod[:take] >> np.uint64(32))
            got += take
            self.pos += take if take == len(x) else take + 1  # a rejected draw is consumed too
        out = np.concatenate(parts) if parts else np.empty(0, np.uint64)
        return (out + np.uint64(lo)).astype(np.int64)


def search_set(n_queries: int, cloud_size: int, sequential: bool = False, repeat: int = 0,
               seed: int = 42) -> np.ndarray:
    """The reference's SearchSet centre indices (inc/benchmarking/search_set.hpp:23-44): one mt19937 seeded
    42 over all repeats; each repeat draws n indices uniform in [0, cloud_size - 1], or with ``sequential``
    one start uniform in [0, cloud_size - n] and the slice after it.  Returns repeat ``repeat``'s row."""
    g = MT19937(seed)
    row = None
    for _ in range(repeat + 1):
        if sequential:
            start = int(g.uniform_int(1, 0, cloud_size - n_queries)[0])
            row = np.arange(start, start + n_queries, dtype=np.int64)
        else:
            row = g.uniform_int(n_queries, 0, cloud_size - 1)
    return row


# The workloads the benchmark and the parity tests use, by name.
CONFIGS = {
    # 1M points, 500 m tile, seed 0, Morton, leaf 128; sphere r = 2.5 and 5.0, 10k centres
    "c1_1M_morton": dict(n=1_000_000, tile_m=500.0, seed=0, encoder=1, max_leaf=128),
    # 10M points, 1.5 km tile, seed 1, Hilbert, leaf 64; r = 1, 2.5, 5; k = 10, 50, 250
    "c2_10M_hilbert": dict(n=10_000_000, tile_m=1500.0, seed=1, encoder=5, max_leaf=64),
}


def config_cloud(name: str, n: int | None = None) -> tuple[np.ndarray, dict]:
    """Cloud of a named configuration; ``n`` scales it down at constant density."""
    cfg = dict(CONFIGS[name])
    if n is not None and n != cfg["n"]:
        cfg["tile_m"] = cfg["tile_m"] * math.sqrt(n / cfg["n"])
        cfg["n"] = n
    xyz = lidar_tile(cfg["n"], cfg["tile_m"], cfg["seed"])
    return xyz, cfg


def batched_clouds(n_clouds: int = 256, seed: int = 2, n_min: int = 10_000, n_max: int = 2_000_000):
    """Cloud descriptors of the multi-cloud (batched) workload: sizes log-uniform
    in [n_min, n_max], density 4-40 points/m^2, Morton or Hilbert, leaf 32/64/128,
    1k-200k query centres each (half radius r ~ U[0.5, 5], half kNN k in {10, 50})."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n_clouds):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        dens = rng.uniform(4.0, 40.0)
        tile = math.sqrt(n / dens)
        out.append(dict(n=n, tile_m=tile, seed=int(rng.integers(0, 2**31 - 1)),
                        encoder=int(rng.choice([1, 5])), max_leaf=int(rng.choice([32, 64, 128])),
                        n_queries=int(rng.integers(1_000, 200_001))))
    return out
