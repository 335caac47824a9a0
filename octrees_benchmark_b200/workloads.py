"""Multi-cloud workloads: many device-resident clouds with their query sets.

``BatchedWorkload`` is the multi-cloud form (clouds of log-uniform sizes,
Morton or Hilbert keys, leaf sizes 32/64/128, each with its own centres: half
radius queries with per-centre radii, half kNN).  Its points come from the
synthetic LiDAR generator; the clouds are generated in a process pool started
with ``spawn`` (the parent may already hold a CUDA context), uploaded and
built one after the other.  The requests it exposes feed the batched engine
(``engine.BatchEngine``); ``sequential`` answers the same requests one cloud
and one call at a time through the single-cloud ABI, the baseline the engine
is compared with.
"""
from __future__ import annotations

import ctypes as C
import math
import multiprocessing as mp
import os
import time

import numpy as np

from . import capi
from .engine import Request
from .linear_octree import LinearOctree
from .synth import batched_clouds, lidar_tile


def _gen(spec):
    return lidar_tile(spec["n"], spec["tile_m"], spec["seed"])


def generate_points(specs, workers: int | None = None):
    """Points of every cloud spec, generated in parallel (spawned workers)."""
    workers = workers or min(len(specs), max(1, (os.cpu_count() or 1)))
    if workers <= 1 or len(specs) < 4:
        return [_gen(s) for s in specs]
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        return pool.map(_gen, specs, chunksize=max(1, len(specs) // (4 * workers)))


class BatchedWorkload:
    """Clouds of ``specs`` (default: the 256-cloud batched set, seed 2) with their requests."""

    def __init__(self, specs=None, device: int = 0, workers: int | None = None, kernel: str = "sphere",
                 algo: str = "neighborsPrune"):
        import torch

        self.specs = specs if specs is not None else batched_clouds()
        t0 = time.perf_counter()
        pts = generate_points(self.specs, workers)
        self.gen_s = time.perf_counter() - t0
        self.clouds = []
        self.requests = []
        self.kernel, self.algo = kernel, algo
        build_s = 0.0
        for ci, (spec, p) in enumerate(zip(self.specs, pts)):
            d = torch.from_numpy(p).cuda(device)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            oc = LinearOctree(d, encoder=spec["encoder"], max_points_leaf=spec["max_leaf"], device=device)
            build_s += time.perf_counter() - t1
            self.clouds.append(oc)
            rng = np.random.default_rng(spec["seed"] ^ 0x5EED)
            nq = spec["n_queries"]
            nr = nq // 2
            nk = nq - nr
            sel = torch.from_numpy(rng.integers(0, spec["n"], nq)).cuda(device)
            centres = d[sel].contiguous()
            radii = torch.from_numpy(rng.uniform(0.5, 5.0, nr)).cuda(device)
            k = int(rng.choice([10, 50]))
            self.requests.append(Request(oc, "radius", centres[:nr], radii=radii, kernel=kernel, algo=algo))
            self.requests.append(Request(oc, "knn", centres[nr:], k=k))
            del d
        self.build_s = build_s
        self.n_points = sum(s["n"] for s in self.specs)
        self.n_queries = sum(s["n_queries"] for s in self.specs)

    def describe(self) -> str:
        sizes = [s["n"] for s in self.specs]
        return (f"{len(self.specs)} synthetic LiDAR clouds (seed 2), sizes log-uniform {min(sizes):,}-{max(sizes):,} "
                f"points ({self.n_points:,} in all), density 4-40 pts/m^2, Morton or Hilbert keys, leaf 32/64/128; "
                f"{self.n_queries:,} centres at cloud points, half radius ({self.kernel}, {self.algo}, per-centre "
                f"r ~ U[0.5, 5] m), half kNN (k in {{10, 50}} per cloud)")

    def sample(self, max_centres: int = 2048):
        """The same requests cut to their first ``max_centres`` centres (autotuning sample)."""
        out = []
        for r in self.requests:
            m = min(int(r.centers.shape[0]), max_centres)
            out.append(Request(r.cloud, r.kind, r.centers[:m], radius=r.radius,
                               radii=None if r.radii is None else r.radii[:m], kernel=r.kernel, algo=r.algo, k=r.k))
        return out


def sequential(wl: BatchedWorkload, stream, out_cap: int, packet: bool, lanes: int = 8, bucket: int = 128):
    """Answer every request with its own single-cloud device call, one after the other on ``stream``.

    Returns (radius results per radius request, (idx, d2) device tensors of the
    last kNN request).  The clouds run on ``stream`` for the duration."""
    import torch

    L = capi.lib()
    MD = capi.OCT_MEM_DEVICE
    dev = torch.cuda.current_device()
    max_nq = max(int(r.centers.shape[0]) for r in wl.requests)
    max_k = max(r.k for r in wl.requests)
    offs = torch.zeros(max_nq + 1, dtype=torch.int64, device=dev)
    idx = torch.empty(max(1, out_cap), dtype=torch.int32, device=dev)
    kidx = torch.empty(max_nq * max_k, dtype=torch.int32, device=dev)
    kd2 = torch.empty(max_nq * max_k, dtype=torch.float64, device=dev)
    kcnt = torch.empty(max_nq, dtype=torch.int32, device=dev)
    tot = C.c_uint64()
    cfg = capi.OctSearchConfig(int(packet), 0, lanes, 0, bucket)
    totals = []
    for oc in wl.clouds:
        capi.check(L.oct_cloud_set_stream(oc.handle, C.c_void_p(stream.cuda_stream)), oc.handle)
        capi.check(L.oct_set_search_config(oc.handle, C.byref(cfg)), oc.handle)
    for r in wl.requests:
        h = r.cloud.handle
        nq = int(r.centers.shape[0])
        if r.kind == "radius":
            st = L.oct_radius_search(h, capi.KERNELS[r.kernel], capi.ALGOS[r.algo], r.centers.data_ptr(), nq,
                                     r.radii.data_ptr() if r.radii is not None else None, r.radius,
                                     offs.data_ptr(), idx.data_ptr(), out_cap, C.byref(tot), MD)
            capi.check(st, h, "sequential radius")
            totals.append(int(tot.value))
        else:
            capi.check(L.oct_knn(h, r.centers.data_ptr(), nq, r.k, kidx.data_ptr(), kd2.data_ptr(), kcnt.data_ptr(),
                                 MD), h, "sequential kNN")
    return totals, kidx, kd2
