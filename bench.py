#!/usr/bin/env python
"""Benchmark of the B200 linear-octree neighbour search.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: a 10,000,000-point synthetic airborne-LiDAR tile (1.5 km x 1.5 km,
seed 1, terrain + canopy cylinders), Hilbert keys, 64 points per leaf.  The
cloud is uploaded, SFC-sorted and its octree built on the device (timed as the
build, in Mpts/s), then every step answers one batch of queries at random
cloud points: 500,000 radius searches (sphere kernel, neighborsPrune, r = 2.5 m,
full CSR output) and 500,000 kNN searches (k = 50).  ``value`` is queries/s
over the whole job (all ranks); the step's inputs are resident in HBM and L2
is flushed before every step.  ``e2e`` is the same step through the engine's
C ABI with host buffers (centres copied in from pinned memory, every result
copied out to pinned memory, inside the timed region); two engines alternate
so that one step's results cross PCIe while the next step computes (the serial
figure is in ``e2e.detail``).  With N GPUs every rank holds its own replica of the cloud and its own
queries (weak scaling, no collective on the data path).

``--impl reference`` times the reference's own CPU implementation (the
reference headers compiled by ``make -C oracle ref``; the oracle's C
restatement if that library is absent) on a bounded sample of the same query
mix with every host thread, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
import traceback

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "queries/s & build Mpts/s at 10M pts, batched vs plain GPU; p99 serve latency"
N_POINTS = 10_000_000
TILE_M = 1500.0
SEED = 1
ENCODER = 5
MAX_LEAF = 64
RADIUS = 2.5
KNN_K = 50
Q_RADIUS = 500_000
Q_KNN = 500_000
L2_FLUSH_BYTES = 512 << 20
# device launches of this library per timed step (counted from an ncu launch list of this bench):
# plain: radius count, 3 scan kernels, fill; kNN.  The packet paths order the queries of each call first
# (keys, histogram scan, 3 sort passes) and search the radius set in one pass (+ 3 scan kernels and the
# chunk compaction), or count and fill with the FP32 filter; kNN in groups adds the fallback launch.
LAUNCHES_PER_STEP = {"plain": 6, "packet": 10 + 7, "packet_fp32": 10 + 7, "knn_per_query": 10 + 6,
                     # engine: epoch, keys, histogram scan, 4 sort passes, one-pass radius, 3 scan kernels,
                     # chunk compaction, request totals, group kNN, fallback kNN
                     "engine": 15}
BUILD_BYTES_PER_POINT = 112  # encode 32 + sort 20 + reorder 52 + leaf counting 8
BUILD_BYTES_PER_NODE = 36    # offsets 4 + ranges 8 + centers 24
# DRAM bytes (read + write) per query of the search kernels, from ncu --set full of this script's
# `--points 6000000 --queries 200000 --search packet --paths packet` case (6M points at this tile's density,
# 200k queries each): k_knn_group k=50 511.8 + 143.8 MB, one-pass k_radius_packet r=2.5 342.3 + 58.8 MB
KNN_DRAM_BYTES_PER_QUERY = (511.8e6 + 143.8e6) / 200_000
RADIUS_DRAM_BYTES_PER_QUERY = (342.3e6 + 58.8e6) / 200_000


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_config(world: int, extra=None):
    cfg = {
        "workload": f"{N_POINTS // 1_000_000}M-point synthetic LiDAR tile ({TILE_M / 1000:g} km, seed {SEED}), "
                    f"Hilbert keys, leaf {MAX_LEAF}; per step {Q_RADIUS} radius queries (sphere, neighborsPrune, "
                    f"r={RADIUS} m, CSR output) + {Q_KNN} kNN queries (k={KNN_K}) at random cloud points",
        "n_points": N_POINTS,
        "queries_per_step": Q_RADIUS + Q_KNN,
        "parallelism": f"replicas x{world}" if world > 1 else "single",
        "l2": "flushed (512 MB write) before every timed step; cloud coordinates 240 MB > L2",
        "data": "synthetic stand-in for the reference's LiDAR clouds (not available offline)",
    }
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------------------ clocks ---
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu), "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            with open(self.path) as f:
                for ln in f:
                    p = [x.strip() for x in ln.split(",")]
                    if len(p) >= 9:
                        rows.append(p)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [s for s in sm if s > 0.5 * (max(sm) if sm else 0)]
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------- CPU baselines ---
def cpu_arm(xyz, threads: int, target_s: float = 10.0):
    """Time the reference CPU implementation on a bounded sample of the query mix.
    Returns a dict describing the baseline and a function running one sample."""
    from octrees_benchmark_b200.synth import query_indices, search_set
    from oracle import oracle as orc

    if orc.reference_available():
        R = orc.Reference(ENCODER, xyz, MAX_LEAF, threads=threads)
        kind = "reference"
        sxyz = R.points()[0]
        cores = R.max_threads() if threads <= 0 else threads

        def run(qr, qk):
            tr, _ = R.time_radius(1, 2, qr, RADIUS, threads)
            tk, _ = R.time_knn(qk, KNN_K, threads)
            return tr, tk

        def ref_radius(qr, kernel=1, algo=2, r=RADIUS):
            return R.radius(kernel, algo, qr, r, threads)

        def ref_knn(qk, k=KNN_K):
            return R.knn(qk, k, threads)
    else:
        P = orc.Port()
        keys, perm, box, sxyz = P.encode_sort(ENCODER, xyz)
        T = P.build(ENCODER, keys, MAX_LEAF, box)
        kind = "port"
        cores = os.cpu_count()

        def run(qr, qk):
            t0 = time.perf_counter()
            T.radius(sxyz, 1, 2, qr, RADIUS)
            t1 = time.perf_counter()
            T.knn(sxyz, qk, KNN_K)
            return t1 - t0, time.perf_counter() - t1

        def ref_radius(qr, kernel=1, algo=2, r=RADIUS):
            return T.radius(sxyz, kernel, algo, qr, r)

        def ref_knn(qk, k=KNN_K):
            return T.knn(sxyz, qk, k)
    # calibrate the sample so that one run is about target_s / 2 of CPU work
    cal = 4000
    q = sxyz[query_indices(2 * cal, len(sxyz), seed=99)]
    tr, tk = run(q[:cal], q[cal:])
    per_q = (tr + tk) / (2 * cal)
    m = int(max(cal, min(Q_RADIUS, target_s / 2 / max(per_q, 1e-9) / 2)))
    sample = sxyz[search_set(2 * m, len(sxyz))]  # the reference's SearchSet stream (mt19937 seeded 42)
    return dict(kind=kind, cores=int(cores), sample_per_kind=m, run=run, sample=sample, sorted_xyz=sxyz,
                ref_radius=ref_radius, ref_knn=ref_knn)


PARITY_QUERIES = 20_000  # per kind: radius and kNN centres of the CPU sample checked on every GPU path


def cpu_leg(args, xyz_h, h, eng, proxy, eng_cfg):
    """The reference CPU path timed on a bounded sample of the step's query mix (all host threads), then the
    first PARITY_QUERIES radius and kNN centres of that sample answered by every GPU search path and compared
    with the reference's answers: neighbour sets (sorted), kNN squared distances (bitwise) and indices (ties at
    the k-th distance by lowest index)."""
    import torch

    from octrees_benchmark_b200 import capi
    from octrees_benchmark_b200.engine import Request
    from tests.parity import csr_set_diffs, knn_diffs

    L = capi.lib()
    MD = capi.OCT_MEM_DEVICE
    arm = cpu_arm(xyz_h, threads=0, target_s=args.cpu_seconds)
    m = arm["sample_per_kind"]
    tr, tk = arm["run"](arm["sample"][:m], arm["sample"][m:])
    cpu = {"value": 2 * m / (tr + tk), "unit": "queries/s", "cores": arm["cores"], "kind": arm["kind"],
           "sample": f"{m} radius (sphere, neighborsPrune, r={RADIUS}) + {m} kNN (k={KNN_K}) queries at random "
                     f"points of the same {N_POINTS:,}-point cloud, all host threads",
           "radius_qps": m / tr, "knn_qps": m / tk}
    p = min(m, PARITY_QUERIES)
    qr_h = np.ascontiguousarray(arm["sample"][:p])
    qk_h = np.ascontiguousarray(arm["sample"][m:m + p])
    t0 = time.perf_counter()
    ro, ri = arm["ref_radius"](qr_h)
    ki, kd, kc = arm["ref_knn"](qk_h)
    ref_s = time.perf_counter() - t0
    sxyz = arm["sorted_xyz"]
    qr, qk = torch.from_numpy(qr_h).cuda(), torch.from_numpy(qk_h).cuda()
    torch.cuda.synchronize()

    def single(packet, fp32, lanes, knn_group):
        cfg = capi.OctSearchConfig(packet, fp32, lanes, knn_group, args.knn_bucket)
        capi.check(L.oct_set_search_config(h, C.byref(cfg)), h, "search config")
        L.oct_search_stats(h, None, None, 1)
        L.oct_knn_filter_stats(h, None, None, None, 1)
        offs = torch.zeros(p + 1, dtype=torch.int64, device="cuda")
        tot = C.c_uint64()
        st = L.oct_radius_search(h, 1, 2, qr.data_ptr(), p, None, RADIUS, offs.data_ptr(), None, 0, C.byref(tot), MD)
        assert st in (capi.OCT_OK, capi.OCT_ERR_CAPACITY)
        out = torch.empty(max(1, tot.value), dtype=torch.int32, device="cuda")
        capi.check(L.oct_radius_search(h, 1, 2, qr.data_ptr(), p, None, RADIUS, offs.data_ptr(), out.data_ptr(),
                                       tot.value, C.byref(tot), MD), h, "parity radius")
        kidx = torch.empty((p, KNN_K), dtype=torch.int32, device="cuda")
        kd2 = torch.empty((p, KNN_K), dtype=torch.float64, device="cuda")
        kcnt = torch.empty(p, dtype=torch.int32, device="cuda")
        capi.check(L.oct_knn(h, qk.data_ptr(), p, KNN_K, kidx.data_ptr(), kd2.data_ptr(), kcnt.data_ptr(), MD), h,
                   "parity kNN")
        capi.check(L.oct_synchronize(h), h)
        tests, retests = C.c_uint64(), C.c_uint64()
        L.oct_search_stats(h, C.byref(tests), C.byref(retests), 1)
        k_tests, k_f64, k_band = C.c_uint64(), C.c_uint64(), C.c_uint64()
        L.oct_knn_filter_stats(h, C.byref(k_tests), C.byref(k_f64), C.byref(k_band), 1)
        band = {"radius_band_hit_fraction": retests.value / tests.value if tests.value else None,
                "knn_band_hit_fraction": k_band.value / k_tests.value if k_tests.value else None}
        return (offs.cpu().numpy(), out[: tot.value].cpu().numpy().view(np.uint32), kidx.cpu().numpy().view(np.uint32),
                kd2.cpu().numpy(), kcnt.cpu().numpy(), band)

    def engine(fp32):
        eng.set_config(**dict(eng_cfg, fp32_filter=fp32))
        try:
            places = eng.run([Request(proxy, "radius", qr, radius=RADIUS, kernel="sphere", algo="neighborsPrune"),
                              Request(proxy, "knn", qk, k=KNN_K)])
            offs, idx = eng.radius_result(places[0])
            kidx, kd2, kcnt = eng.knn_result(places[1], KNN_K)
        finally:
            eng.set_config(**eng_cfg)
        return offs, idx, kidx, kd2, kcnt, {}

    runs = {"plain": lambda: single(0, 0, args.radius_group, 0), "packet": lambda: single(1, 0, 8, 1),
            "packet_fp32": lambda: single(1, 1, 8, 1), "packet_fp32_radius": lambda: single(1, 2, 8, 1),
            "engine": lambda: engine(0), "engine_fp32": lambda: engine(1), "engine_fp32_radius": lambda: engine(2)}
    out = {}
    total_diffs, max_err = 0, 0.0
    for name, fn in runs.items():
        offs, idx, kidx, kd2, kcnt, band = fn()
        rd = csr_set_diffs(offs, idx, ro, ri)
        kdiff, kerr, ties = knn_diffs(kidx, kd2, kcnt, ki, kd, kc, sxyz, qk_h)
        out[name] = dict(radius_set_diffs=rd, knn_diffs=kdiff, max_d2_err=kerr, knn_tie_groups_checked=ties,
                         radius_neighbours=int(offs[-1]), **band)
        total_diffs += rd + kdiff
        max_err = max(max_err, kerr)
    cfg0 = capi.OctSearchConfig(1, 0, 8, 1, args.knn_bucket)  # the headline path's configuration again
    capi.check(L.oct_set_search_config(h, C.byref(cfg0)), h, "search config")
    parity = {"against": arm["kind"], "centres": {"radius": p, "knn": p},
              "query": f"sphere neighborsPrune r={RADIUS} m and kNN k={KNN_K} at the CPU sample's centres",
              "set_diffs": total_diffs, "max_d2_err": max_err, "paths": out, "reference_s": ref_s,
              "rule": "radius: sorted neighbour index sets equal; kNN: counts and squared distances bitwise equal, "
                      "index sets equal below the k-th distance, ties at the k-th distance the lowest indices"}
    return {"cpu": cpu, "parity": parity}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    from octrees_benchmark_b200.synth import lidar_tile

    xyz = lidar_tile(N_POINTS, TILE_M, SEED)
    arm = cpu_arm(xyz, threads=0, target_s=args.cpu_seconds)
    m = arm["sample_per_kind"]
    q = arm["sample"]
    for _ in range(args.warmup):
        arm["run"](q[:m], q[m:])
    times = []
    for _ in range(args.steps):
        tr, tk = arm["run"](q[:m], q[m:])
        times.append(tr + tk)
    total = sum(times)
    value = 2 * m * args.steps / total
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(1, {"sample": f"{m} radius + {m} kNN queries per step (bounded CPU sample)"}),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": arm["cores"], "kind": arm["kind"],
                         "sample": f"{m} radius + {m} kNN queries of the same mix per step"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------ multi-cloud batch ---
def run_batched(args, dev):
    """256 clouds with their own query sets: one engine batch against sequential per-cloud calls."""
    import torch

    from octrees_benchmark_b200.engine import BatchEngine
    from octrees_benchmark_b200.workloads import BatchedWorkload, sequential

    wl = BatchedWorkload(device=dev)
    eng = BatchEngine(device=dev)
    tune = eng.autotune(wl.sample(4096))
    for _ in range(args.warmup):
        places = eng.run(wl.requests)
    dev_ms, wall_ms = [], []
    for _ in range(args.batched_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        places = eng.run(wl.requests)
        wall_ms.append(1e3 * (time.perf_counter() - t0))
        dev_ms.append(eng.last_ms)
    radius_totals = [pl.n_results for pl, r in zip(places, wl.requests) if r.kind == "radius"]
    n_results = sum(radius_totals)
    out_cap = max(radius_totals) + 1024
    eng_kidx, eng_kd2, _ = eng.knn_result(places[-1], wl.requests[-1].k)
    del eng
    torch.cuda.empty_cache()
    seq = {}
    stream = torch.cuda.Stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, packet in (("sequential_plain", False), ("sequential_packet", True)):
        sequential(wl, stream, out_cap, packet)  # warm-up (first call of each cloud sizes its scratch)
        times = []
        for _ in range(args.batched_steps):
            stream.synchronize()
            ev0.record(stream)
            totals, kidx, kd2 = sequential(wl, stream, out_cap, packet)
            ev1.record(stream)
            stream.synchronize()
            times.append(ev0.elapsed_time(ev1))
        # the same results as the batch: every radius request's count, the last kNN request's pairs
        assert totals == radius_totals, f"{name}: radius result counts differ from the batch"
        nk, k = int(wl.requests[-1].centers.shape[0]), wl.requests[-1].k
        assert np.array_equal(kidx[: nk * k].cpu().numpy().view(np.uint32).reshape(nk, k), eng_kidx)
        assert np.array_equal(kd2[: nk * k].cpu().numpy().reshape(nk, k), eng_kd2)
        seq[name] = {"ms": statistics.median(times), "qps": wl.n_queries / (statistics.median(times) / 1e3)}
    b_ms = statistics.median(dev_ms)
    return {
        "workload": wl.describe(),
        "queries": wl.n_queries, "radius_results": n_results,
        "batched_ms": b_ms, "batched_wall_ms": statistics.median(wall_ms), "batched_qps": wl.n_queries / (b_ms / 1e3),
        "sequential_plain_ms": seq["sequential_plain"]["ms"], "sequential_plain_qps": seq["sequential_plain"]["qps"],
        "sequential_packet_ms": seq["sequential_packet"]["ms"],
        "sequential_packet_qps": seq["sequential_packet"]["qps"],
        "speedup_vs_sequential_plain": seq["sequential_plain"]["ms"] / b_ms,
        "speedup_vs_sequential_packet": seq["sequential_packet"]["ms"] / b_ms,
        "autotuned": tune, "steps": args.batched_steps, "warmup": args.warmup,
        "timing": "batch: CUDA events around the engine's whole device sequence (descriptor copy to summary copy); "
                  "sequential: CUDA events around all 512 calls on one stream, host syncs of the calls included",
        "generate_s": wl.gen_s, "build_all_clouds_s": wl.build_s,
        "parity": "every radius request's result count and the last kNN request's pairs equal between batch and "
                  "sequential calls (full bitwise parity is in the GPU tests)",
    }


# ----------------------------------------------------------- large skewed cloud ---
def run_large(args, dev):
    """500M points on a 10 km tile (rural 5 pts/m^2 + urban building clusters ~2000 pts/m^2), built from HBM;
    10M radius centres (r = 2.5 m, counts) and 10M kNN centres (k = 1000, in batches) on the FP32-filter
    configuration; a 1% sample of each compared with the plain FP64 path."""
    import torch

    from octrees_benchmark_b200 import capi
    from octrees_benchmark_b200.synth import large_tile_device

    L = capi.lib()
    MD = capi.OCT_MEM_DEVICE
    n = args.large_points
    t0 = time.perf_counter()
    xyz = large_tile_device(n)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    p = capi.OctParams(64, ENCODER, dev, 0)
    h = C.c_void_p()
    capi.check(L.oct_cloud_create(C.byref(p), C.byref(h)), None, "create")
    info = capi.OctTreeInfo()
    bt = []
    for rep in range(3):
        capi.check(L.oct_set_points(h, xyz.data_ptr(), n, MD), h)
        capi.check(L.oct_synchronize(h), h)
        t1 = time.perf_counter()
        capi.check(L.oct_encode_sort(h, None, None, None, None, MD), h)
        capi.check(L.oct_build(h, C.byref(info)), h)
        torch.cuda.synchronize()
        if rep:
            bt.append(time.perf_counter() - t1)
    build_s = min(bt)
    peak, _ = measured_peak()
    build_bytes = BUILD_BYTES_PER_POINT * n + BUILD_BYTES_PER_NODE * info.n_total
    g = torch.Generator(device="cuda").manual_seed(30)
    nq = args.large_queries
    qr = xyz[torch.randint(0, n, (nq,), device="cuda", generator=g)].contiguous()
    qk = xyz[torch.randint(0, n, (nq,), device="cuda", generator=g)].contiguous()
    del xyz
    torch.cuda.empty_cache()
    stream = torch.cuda.Stream()
    capi.check(L.oct_cloud_set_stream(h, C.c_void_p(stream.cuda_stream)), h)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def config(packet, fp32):
        cfg = capi.OctSearchConfig(packet, fp32, 8, 0, 256)
        capi.check(L.oct_set_search_config(h, C.byref(cfg)), h)

    # radius r = 2.5 m: neighbour counts of every centre, FP32 filter + FP64 band
    config(1, 1)
    counts = torch.empty(nq, dtype=torch.int64, device="cuda")
    L.oct_search_stats(h, None, None, 1)
    capi.check(L.oct_radius_count(h, 1, 2, qr.data_ptr(), min(nq, 100_000), None, RADIUS, counts.data_ptr(), MD), h)
    ev0.record(stream)
    capi.check(L.oct_radius_count(h, 1, 2, qr.data_ptr(), nq, None, RADIUS, counts.data_ptr(), MD), h)
    ev1.record(stream)
    capi.check(L.oct_synchronize(h), h)
    rad_ms = ev0.elapsed_time(ev1)
    tests, retests = C.c_uint64(), C.c_uint64()
    L.oct_search_stats(h, C.byref(tests), C.byref(retests), 1)
    total_nbrs = int(counts.sum().item())
    # the same counts in FP64 (no filter), for the FP32 filter's effect on a cloud far larger than L2
    config(1, 0)
    counts64 = torch.empty(nq, dtype=torch.int64, device="cuda")
    ev0.record(stream)
    capi.check(L.oct_radius_count(h, 1, 2, qr.data_ptr(), nq, None, RADIUS, counts64.data_ptr(), MD), h)
    ev1.record(stream)
    capi.check(L.oct_synchronize(h), h)
    rad64_ms = ev0.elapsed_time(ev1)
    counts_equal = bool(torch.equal(counts, counts64))
    del counts64
    config(1, 1)
    # kNN k = 1000 in batches (the outputs of all 10M centres would be 120 GB)
    K = args.large_k
    kb = min(nq, 1_000_000)
    kidx = torch.empty((kb, K), dtype=torch.int32, device="cuda")
    kd2 = torch.empty((kb, K), dtype=torch.float64, device="cuda")
    knn_ms = 0.0
    for s in range(0, nq, kb):
        m = min(kb, nq - s)
        ev0.record(stream)
        capi.check(L.oct_knn(h, qk[s:].data_ptr(), m, K, kidx.data_ptr(), kd2.data_ptr(), None, MD), h, "large kNN")
        ev1.record(stream)
        capi.check(L.oct_synchronize(h), h)
        knn_ms += ev0.elapsed_time(ev1)
    # parity on a 1 % sample: FP32-filter configuration against the plain FP64 path
    ns = max(1, nq // 100)

    def radius_csr(packet, fp32):
        config(packet, fp32)
        offs = torch.zeros(ns + 1, dtype=torch.int64, device="cuda")
        tot = C.c_uint64()
        st = L.oct_radius_search(h, 1, 2, qr.data_ptr(), ns, None, RADIUS, offs.data_ptr(), None, 0, C.byref(tot), MD)
        assert st in (capi.OCT_OK, capi.OCT_ERR_CAPACITY)
        out = torch.empty(max(1, tot.value), dtype=torch.int32, device="cuda")
        capi.check(L.oct_radius_search(h, 1, 2, qr.data_ptr(), ns, None, RADIUS, offs.data_ptr(), out.data_ptr(),
                                       tot.value, C.byref(tot), MD), h)
        capi.check(L.oct_synchronize(h), h)
        return offs, out[: tot.value]

    def knn_sample(packet):
        config(packet, 0)
        i = torch.empty((ns, K), dtype=torch.int32, device="cuda")
        d = torch.empty((ns, K), dtype=torch.float64, device="cuda")
        capi.check(L.oct_knn(h, qk.data_ptr(), ns, K, i.data_ptr(), d.data_ptr(), None, MD), h)
        capi.check(L.oct_synchronize(h), h)
        return i, d

    o1, i1 = radius_csr(1, 1)
    o2, i2 = radius_csr(0, 0)
    radius_same = bool(torch.equal(o1, o2) and torch.equal(i1, i2))
    sample_nbrs = int(o1[-1].item())
    del i1, i2
    a1, d1 = knn_sample(1)
    a2, d2 = knn_sample(0)
    knn_same_d2 = bool(torch.equal(d1, d2))
    knn_same_idx = bool(torch.equal(a1, a2))
    L.oct_cloud_destroy(h)
    return {
        "workload": f"{n:,} points on a {10:g} km tile (seed 3, generated on the device): rural ground 5 pts/m^2 "
                    f"(60 %), 50 urban building clusters of radius 10-40 m (~2000 pts/m^2, 40 %); Hilbert, leaf 64; "
                    f"{nq:,} radius centres (sphere, neighborsPrune, r={RADIUS} m, FP32 filter + FP64 band, neighbour "
                    f"counts) and {nq:,} kNN centres (k={K}, batches of {kb:,}) at random cloud points",
        "build_ms": 1e3 * build_s, "build_mpts_s": n / build_s / 1e6,
        "build_frac_of_hbm": build_bytes / build_s / 1e9 / peak, "nodes": info.n_total, "depth": info.max_depth_seen,
        "radius_ms": rad_ms, "radius_qps": nq / (rad_ms / 1e3), "radius_neighbours": total_nbrs,
        "radius_fp64_ms": rad64_ms, "radius_fp32_vs_fp64": rad64_ms / rad_ms, "radius_counts_equal_fp64": counts_equal,
        "radius_neighbours_per_s": total_nbrs / (rad_ms / 1e3),
        "band_hit_fraction": retests.value / tests.value if tests.value else None,
        "knn_ms": knn_ms, "knn_qps": nq / (knn_ms / 1e3),
        "parity_sample": {"centres": ns, "radius_neighbours": sample_nbrs, "radius_csr_equal_plain": radius_same,
                          "knn_d2_equal_plain": knn_same_d2, "knn_idx_equal_plain": knn_same_idx},
        "generate_s": gen_s,
        "timing": "build: wall clock of encode + sort + reorder + octree from points in HBM (best of 2 after a "
                  "warm-up); radius and kNN: CUDA events around the calls on the cloud's stream",
    }


# ------------------------------------------------------------------ serving ---
def run_serving(args, dev):
    """The serving stream replayed in real time: the batching server, then the plain one-request-per-launch one."""
    from octrees_benchmark_b200.serve import Server, ServingWorkload, replay

    wl = ServingWorkload(device=dev, seconds=args.serve_seconds)
    clocks = ClockSampler(dev)
    clocks.start()
    srv = Server(device=dev, slots=args.serve_slots, max_batch_queries=args.serve_max_batch,
                 max_wait_ms=args.serve_max_wait, fifo=args.serve_fifo, graph=not args.serve_no_graph)
    try:
        batched = replay(wl, srv, drain_s=args.serve_drain)
    finally:
        srv.close()
        clk = clocks.stop()
    srv = Server(device=dev, plain=True)
    try:
        plain = replay(wl, srv, drain_s=args.serve_drain)
    finally:
        srv.close()
    return {
        "workload": wl.describe(),
        "batched": batched, "plain": plain,
        "p50_ms": batched["p50_ms"], "p99_ms": batched["p99_ms"], "qps": batched["qps"],
        "p99_vs_plain": (plain["p99_ms"] / batched["p99_ms"]) if batched["p99_ms"] and plain["p99_ms"] else None,
        "qps_vs_plain": (batched["qps"] / plain["qps"]) if plain["qps"] else None,
        "clocks_batched": clk,
        "timing": "latency = submit to results complete on the device (scheduler clock); qps = centres answered / "
                  "wall time from the first arrival to the last completion; a server still busy "
                  f"{args.serve_drain:g} s after the stream ends is stopped and its unanswered requests reported",
        "generate_s": wl.gen_s,
    }


# --------------------------------------------------------------- B200 arm ---
def run_b200(args, rank, world, local_rank):
    import torch

    from octrees_benchmark_b200 import capi
    from octrees_benchmark_b200.synth import lidar_tile

    L = capi.lib()
    dev = local_rank
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    xyz_h = lidar_tile(N_POINTS, TILE_M, SEED)
    xyz_d = torch.from_numpy(xyz_h).cuda()
    p = capi.OctParams(MAX_LEAF, ENCODER, dev, capi.OCT_CLOUD_SORT_8PASS if args.sort_8pass else 0)
    h = C.c_void_p()
    capi.check(L.oct_cloud_create(C.byref(p), C.byref(h)), None, "create")
    capi.check(L.oct_cloud_set_stream(h, C.c_void_p(stream.cuda_stream)), h)
    capi.check(L.oct_set_radius_group(h, args.radius_group), h)
    info = capi.OctTreeInfo()
    MD = capi.OCT_MEM_DEVICE

    # ---- build from points resident in HBM: bbox + encode + sort + reorder + octree ----
    # (the upload into the cloud, a device-to-device copy, is timed separately)
    def build_once():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        capi.check(L.oct_set_points(h, xyz_d.data_ptr(), N_POINTS, MD), h, "set_points")
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        capi.check(L.oct_encode_sort(h, None, None, None, None, MD), h, "encode_sort")
        capi.check(L.oct_build(h, C.byref(info)), h, "build")
        torch.cuda.synchronize()
        return t1 - t0, time.perf_counter() - t1

    for _ in range(max(1, args.warmup)):
        build_once()
    bt, ut = [], []
    for _ in range(args.steps):
        u_, b_ = build_once()
        ut.append(u_)
        bt.append(b_)
    build_s = statistics.median(bt)
    upload_s = statistics.median(ut)

    # sorted cloud on the device, query centres = random cloud points
    sorted_xyz = torch.empty((N_POINTS, 3), dtype=torch.float64, device="cuda")
    capi.check(L.oct_encode_sort(h, None, None, None, sorted_xyz.data_ptr(), MD), h)
    capi.check(L.oct_build(h, C.byref(info)), h)
    torch.cuda.synchronize()
    gen = torch.Generator(device="cuda")
    n_batches = args.steps + args.warmup
    batches = []
    for b in range(n_batches):
        gen.manual_seed(1000 * rank + b)
        ir = torch.randint(0, N_POINTS, (Q_RADIUS,), device="cuda", generator=gen)
        ik = torch.randint(0, N_POINTS, (Q_KNN,), device="cuda", generator=gen)
        batches.append((sorted_xyz[ir].contiguous(), sorted_xyz[ik].contiguous()))
    offs = torch.zeros(Q_RADIUS + 1, dtype=torch.int64, device="cuda")
    tot = C.c_uint64()
    st = L.oct_radius_search(h, 1, 2, batches[0][0].data_ptr(), Q_RADIUS, None, RADIUS, offs.data_ptr(), None, 0,
                             C.byref(tot), MD)
    assert st in (capi.OCT_OK, capi.OCT_ERR_CAPACITY)
    cap = int(tot.value * 1.5) + 1024
    idx_out = torch.empty(cap, dtype=torch.int32, device="cuda")
    kidx = torch.empty((Q_KNN, KNN_K), dtype=torch.int32, device="cuda")
    kd2 = torch.empty((Q_KNN, KNN_K), dtype=torch.float64, device="cuda")
    kcnt = torch.empty(Q_KNN, dtype=torch.int32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    # (packet, fp32_filter, lanes, kNN in groups of 4 queries per warp)
    # (packet, fp32_filter, lanes, knn_packet); fp32_filter 1: the radius and kNN FP32 filters, 2: radius only
    SEARCH_PATHS = {"plain": (0, 0, args.radius_group, 0), "packet": (1, 0, 8, 1), "packet_fp32": (1, 1, 8, 1),
                    "packet_fp32_radius": (1, 2, 8, 1), "knn_per_query": (1, 0, 8, 0), "engine": (1, 0, 8, 1),
                    "engine_fp32": (1, 1, 8, 1), "engine_fp32_radius": (1, 2, 8, 1)}

    # the batched engine: both request sets of a step in one graph launch (kNN beside the radius search)
    from types import SimpleNamespace

    from octrees_benchmark_b200.engine import BatchEngine, Request

    proxy = SimpleNamespace(handle=h)
    eng = BatchEngine(device=dev, reserve_results=cap)
    eng_reqs = [[Request(proxy, "radius", qr, radius=RADIUS, kernel="sphere", algo="neighborsPrune"),
                 Request(proxy, "knn", qk, k=KNN_K)] for qr, qk in batches]
    wanted = [p_ for p_ in args.paths.split(",") if p_] if args.paths else ["engine"]
    # the engine is autotuned when an engine path runs (a profile of the single-cloud kernels skips it)
    eng_cfg = eng.autotune(eng_reqs[0]) if args.search == "engine" or any(
        p_.startswith("engine") for p_ in wanted) else eng.config()

    def engine_step(b):
        with torch.cuda.stream(stream):
            flush.zero_()
        stream.synchronize()
        places = eng.run(eng_reqs[b])
        ms = eng.last_ms
        return None, ms, 0.0, int(places[0].n_results)

    def configure(name):
        if name.startswith("engine"):  # the batched engine: its autotuned configuration, FP32 filters as named
            eng.set_config(**dict(eng_cfg, fp32_filter={"engine_fp32": 1, "engine_fp32_radius": 2}.get(
                name, eng_cfg["fp32_filter"])))
        packet, fp32, lanes, knn_packet = SEARCH_PATHS[name]
        cfg = capi.OctSearchConfig(packet, fp32, lanes, knn_packet, args.knn_bucket)
        capi.check(L.oct_set_search_config(h, C.byref(cfg)), h, "search config")

    def step(b):
        qr, qk = batches[b]
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[0].record(stream)
            L.oct_search_timing(h, 0)  # the kernel times cover the search calls below, not this count-only call
            capi.check(L.oct_radius_count(h, 1, 2, qr.data_ptr(), Q_RADIUS, None, RADIUS, offs.data_ptr(), MD), h)
            L.oct_search_timing(h, 1)
            ev[1].record(stream)
            capi.check(L.oct_radius_search(h, 1, 2, qr.data_ptr(), Q_RADIUS, None, RADIUS, offs.data_ptr(),
                                           idx_out.data_ptr(), cap, C.byref(tot), MD), h, "radius_search")
            ev[2].record(stream)
            capi.check(L.oct_knn(h, qk.data_ptr(), Q_KNN, KNN_K, kidx.data_ptr(), kd2.data_ptr(), kcnt.data_ptr(),
                                 MD), h, "knn")
            ev[3].record(stream)
        stream.synchronize()
        return ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3]), int(tot.value)

    clocks = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0])
                          if os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[0].isdigit() else dev)
    paths = {}
    clocks.start()
    run_paths = [p_ for p_ in SEARCH_PATHS if not args.paths or p_ in args.paths.split(",") or p_ == args.search]
    for name in run_paths:
        configure(name)
        run_step = engine_step if name.startswith("engine") else step
        for b in range(args.warmup):
            run_step(b)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        L.oct_search_stats(h, None, None, 1)
        L.oct_knn_filter_stats(h, None, None, None, 1)
        L.oct_search_timing(h, 1)  # CUDA events around the search kernels themselves (single-cloud paths)
        L.oct_search_kernel_times(h, None, None, None, None, 1)
        t_count = t_search = t_knn = 0.0
        nbrs = 0
        for s in range(args.steps):
            a_, b_, c_, tt = run_step(args.warmup + s)
            t_count += a_ or 0.0
            t_search += b_
            t_knn += c_
            nbrs += tt
        torch.cuda.synchronize()
        kr_ms, kr_n, kk_ms, kk_n = C.c_double(), C.c_uint64(), C.c_double(), C.c_uint64()
        L.oct_search_kernel_times(h, C.byref(kr_ms), C.byref(kr_n), C.byref(kk_ms), C.byref(kk_n), 1)
        L.oct_search_timing(h, 0)
        tests, retests = C.c_uint64(), C.c_uint64()
        L.oct_search_stats(h, C.byref(tests), C.byref(retests), 1)
        k_tests, k_f64, k_band = C.c_uint64(), C.c_uint64(), C.c_uint64()
        L.oct_knn_filter_stats(h, C.byref(k_tests), C.byref(k_f64), C.byref(k_band), 1)
        step_ms = (t_search + t_knn) / args.steps  # the count-only call is a separate measurement
        tmax = torch.tensor([step_ms, t_search / args.steps, t_knn / args.steps], dtype=torch.float64, device="cuda")
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.all_reduce(tmax, op=torch.distributed.ReduceOp.MAX)
        step_ms, rad_ms, knn_ms = (float(v) for v in tmax.tolist())
        if name.startswith("engine"):  # radius and kNN overlap: one device time for the whole batch
            rad_ms = knn_ms = float("nan")
        paths[name] = {"ms_per_step": step_ms, "qps": world * (Q_RADIUS + Q_KNN) / (step_ms / 1e3),
                       "radius_qps": world * Q_RADIUS / (rad_ms / 1e3) if rad_ms == rad_ms else None,
                       "knn_qps": world * Q_KNN / (knn_ms / 1e3) if knn_ms == knn_ms else None,
                       "radius_ms": rad_ms if rad_ms == rad_ms else None, "knn_ms": knn_ms if knn_ms == knn_ms else None,
                       "radius_count_only_ms": t_count / args.steps if not name.startswith("engine") else None,
                       "avg_neighbours": nbrs / args.steps / Q_RADIUS, "nbrs_per_step": nbrs / args.steps,
                       "point_tests": tests.value, "fp64_retests": retests.value,
                       "band_hit_fraction": (retests.value / tests.value) if tests.value else None,
                       # the group kNN's FP32 filter: FP32 point tests, the FP64 tests they leave
                       # (candidates + band), band hits (FP64 tests of points that then fail)
                       "knn_fp32_tests": k_tests.value, "knn_fp64_tests": k_f64.value,
                       "knn_band_hit_fraction": (k_band.value / k_tests.value) if k_tests.value else None,
                       # device time of the search kernels alone (CUDA events on the cloud's stream around each
                       # k_radius_packet / k_knn_group launch), per launch; every launch answers one step's queries
                       "kernel_ms": {"k_radius_packet": kr_ms.value / kr_n.value if kr_n.value else None,
                                     "k_knn_group": kk_ms.value / kk_n.value if kk_n.value else None,
                                     "launches": [kr_n.value, kk_n.value]}}
    clk = clocks.stop()
    chosen = paths[args.search]
    configure(args.search)
    step_ms_max = chosen["ms_per_step"]
    value = chosen["qps"]

    # ---- e2e through the host-buffer ABI (pinned buffers, copies in the timed region) ----
    e2e_val = None
    e2e_detail = None
    h2d = d2h = 0
    if not args.no_e2e and args.search == "engine":
        # Through the engine's public API (oct_engine_submit / oct_engine_wait / oct_engine_copy_*): every step's
        # centres copied in from pinned host memory and every result copied out to pinned host memory, all inside
        # the timed region.  Serial: one engine, copy in -> run -> copy out.  Pipelined (the reported value): two
        # engines on their own streams alternate, so step s's results cross PCIe while step s+1 computes; the
        # timed region covers the whole sequence, the pipeline's fill and drain included.
        n_all = args.warmup + args.steps
        qrh_all = [torch.empty((Q_RADIUS, 3), dtype=torch.float64).pin_memory() for _ in range(n_all)]
        qkh_all = [torch.empty((Q_KNN, 3), dtype=torch.float64).pin_memory() for _ in range(n_all)]
        for s_ in range(n_all):
            qrh_all[s_].copy_(batches[s_][0])
            qkh_all[s_].copy_(batches[s_][1])
        offs_h = torch.empty(Q_RADIUS + 1, dtype=torch.int64).pin_memory().numpy()
        idx_h = torch.empty(cap, dtype=torch.int32).pin_memory().numpy()
        kidx_h = torch.empty((Q_KNN, KNN_K), dtype=torch.int32).pin_memory().numpy()
        kd2_h = torch.empty((Q_KNN, KNN_K), dtype=torch.float64).pin_memory().numpy()
        kcnt_h = torch.empty(Q_KNN, dtype=torch.int32).pin_memory().numpy()
        L_ = capi.lib()
        eng2 = BatchEngine(device=dev, reserve_results=cap)
        eng2.set_config(**eng_cfg)
        engs = [eng, eng2]
        # three device input sets: step s reads set s % 3, so the next step's centres are copied in while the
        # step before is still computing (its own set) and the one before that has its results copied out
        dbufs = [(torch.empty((Q_RADIUS, 3), dtype=torch.float64, device="cuda"),
                  torch.empty((Q_KNN, 3), dtype=torch.float64, device="cuda")) for _ in range(3)]
        reqs_e2e = [[Request(proxy, "radius", qrd, radius=RADIUS, kernel="sphere", algo="neighborsPrune"),
                     Request(proxy, "knn", qkd, k=KNN_K)] for qrd, qkd in dbufs]
        in_ev = [torch.cuda.Event() for _ in range(3)]
        torch.cuda.synchronize()

        def copy_in_async(s_):
            qrd, qkd = dbufs[s_ % 3]
            with torch.cuda.stream(stream):
                qrd.copy_(qrh_all[s_], non_blocking=True)
                qkd.copy_(qkh_all[s_], non_blocking=True)
                in_ev[s_ % 3].record(stream)

        def copy_in(s_, slot=None):
            copy_in_async(s_)
            in_ev[s_ % 3].synchronize()

        def copy_out(e):
            pl = e.wait()
            capi.check(L_.oct_engine_copy_radius(e._h, C.byref(pl[0]), offs_h.ctypes.data, idx_h.ctypes.data, cap,
                                                 0), None, "e2e copy radius")
            capi.check(L_.oct_engine_copy_knn(e._h, C.byref(pl[1]), KNN_K, kidx_h.ctypes.data, kd2_h.ctypes.data,
                                              kcnt_h.ctypes.data, 0), None, "e2e copy kNN")
            return pl

        copy_out_s = []  # wall time of each copy-out call inside the timed pipelined run

        def timed_copy_out(e, record):
            t0_ = time.perf_counter()
            pl_ = copy_out(e)
            if record:
                copy_out_s.append(time.perf_counter() - t0_)
            return pl_

        def pipelined(first, count, record=False):
            # step j: its centres are already in (copied while step j - 1 ran), submit it, start copying step
            # j + 1's centres in (set (j + 1) % 3: step j - 2 used it and its results are out), then copy step
            # j - 1's results out while step j computes
            copy_in_async(first)
            for j in range(count):
                slot = j % 2
                in_ev[(first + j) % 3].synchronize()
                engs[slot].submit(reqs_e2e[(first + j) % 3])
                if j + 1 < count:
                    copy_in_async(first + j + 1)
                if j > 0:
                    timed_copy_out(engs[1 - slot], record)
            return timed_copy_out(engs[(count - 1) % 2], record)

        et = []  # serial steps
        for s_ in range(n_all):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            copy_in(s_)
            eng.submit(reqs_e2e[s_ % 3])
            pl = copy_out(eng)
            t1 = time.perf_counter()
            if s_ >= args.warmup:
                et.append(t1 - t0)
        pipelined(0, args.warmup)  # engine 2's graphs captured, both warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pl = pipelined(args.warmup, args.steps, record=True)
        t_pipe = (time.perf_counter() - t0) / args.steps
        h2d = 24 * (Q_RADIUS + Q_KNN)
        d2h = 8 * (Q_RADIUS + 1) + 4 * int(pl[0].n_results) + Q_KNN * KNN_K * 12 + 4 * Q_KNN
        e2e_t = torch.tensor([t_pipe], dtype=torch.float64, device="cuda")
        if world > 1:
            torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
        e2e_val = world * (Q_RADIUS + Q_KNN) / float(e2e_t.item())
        e2e_detail = {"api": "oct_engine_submit / oct_engine_wait + oct_engine_copy_radius / oct_engine_copy_knn",
                      "pipelined_step_ms": round(1e3 * t_pipe, 3),
                      # one step's copy-out call (455 MB at this size), the step's floor once the link is busy
                      "copy_out_ms_median": round(1e3 * statistics.median(copy_out_s), 3) if copy_out_s else None,
                      "serial_step_ms_all": [round(1e3 * v, 2) for v in et],
                      "serial_qps": world * (Q_RADIUS + Q_KNN) / statistics.median(et),
                      "timing": "wall clock over the timed steps; pipelined: two engines alternate (each step's "
                                "results copied out while the next step computes and the one after is copied in), "
                                "fill and drain included"}
        eng2.close()
    elif not args.no_e2e:
        qrh = torch.empty((Q_RADIUS, 3), dtype=torch.float64).pin_memory().numpy()
        qkh = torch.empty((Q_KNN, 3), dtype=torch.float64).pin_memory().numpy()
        offs_h = torch.empty(Q_RADIUS + 1, dtype=torch.int64).pin_memory().numpy()
        idx_h = torch.empty(cap, dtype=torch.int32).pin_memory().numpy()
        kidx_h = torch.empty((Q_KNN, KNN_K), dtype=torch.int32).pin_memory().numpy()
        kd2_h = torch.empty((Q_KNN, KNN_K), dtype=torch.float64).pin_memory().numpy()
        kcnt_h = torch.empty(Q_KNN, dtype=torch.int32).pin_memory().numpy()
        et, er, ek = [], [], []
        for s in range(args.warmup + args.steps):
            qr, qk = batches[s]
            qrh[:] = qr.cpu().numpy()
            qkh[:] = qk.cpu().numpy()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            capi.check(L.oct_radius_search(h, 1, 2, qrh.ctypes.data, Q_RADIUS, None, RADIUS, offs_h.ctypes.data,
                                           idx_h.ctypes.data, cap, C.byref(tot), 0), h, "e2e radius")
            tm = time.perf_counter()
            capi.check(L.oct_knn(h, qkh.ctypes.data, Q_KNN, KNN_K, kidx_h.ctypes.data, kd2_h.ctypes.data,
                                 kcnt_h.ctypes.data, 0), h, "e2e knn")
            t1 = time.perf_counter()
            if s >= args.warmup:
                et.append(t1 - t0)
                er.append(tm - t0)
                ek.append(t1 - tm)
                h2d = 24 * (Q_RADIUS + Q_KNN)
                d2h = 8 * (Q_RADIUS + 1) + 4 * int(tot.value) + Q_KNN * KNN_K * 12 + 4 * Q_KNN
        e2e_t = torch.tensor([statistics.median(et)], dtype=torch.float64, device="cuda")
        if world > 1:
            torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
        e2e_val = world * (Q_RADIUS + Q_KNN) / float(e2e_t.item())
        # the box's device-to-host bandwidth into pinned memory, for reading e2e
        probe = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        probe_h = torch.empty(256 << 20, dtype=torch.uint8).pin_memory()
        probe_h.copy_(probe)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        probe_h.copy_(probe)
        torch.cuda.synchronize()
        d2h_gbs = (256 << 20) / (time.perf_counter() - t0) / 1e9
        e2e_detail = {"radius_ms": 1e3 * statistics.median(er), "knn_ms": 1e3 * statistics.median(ek),
                      "step_ms_all": [round(1e3 * v, 2) for v in et], "pinned_d2h_gbs": d2h_gbs}

    # ---- roofline of the dominant kernel of the chosen path ----
    peak, peak_kind = measured_peak()
    rad_bytes = 24 * Q_RADIUS + 28 * chosen["nbrs_per_step"]
    knn_bytes = (24 + 36 * KNN_K) * Q_KNN
    # per-kernel times: the engine runs the packet path's kernels side by side, so they are timed there alone
    kpath = args.search if chosen["radius_ms"] is not None else ("packet" if "packet" in paths else args.search)
    km = paths[kpath].get("kernel_ms") or {}
    rad_ms, knn_ms = km.get("k_radius_packet"), km.get("k_knn_group")
    if rad_ms is None or knn_ms is None:  # only the engine path ran: its kernels overlap, no per-kernel time
        rad_ms = knn_ms = float("nan")
    # each time is the kernel's own launch on the cloud's stream (CUDA events around the launch), averaged over
    # the timed steps' launches; one launch answers one step's queries of its kind
    rad = {"kernel": f"k_radius_packet (neighborsPrune sphere r={RADIUS}, one pass, {kpath} path)", "ms": rad_ms,
           "achieved": rad_bytes / (rad_ms / 1e3) / 1e9,
           "call_ms": paths[kpath]["radius_ms"]}
    knn = {"kernel": f"k_knn_group (k={KNN_K}, {kpath} path)", "ms": knn_ms,
           "achieved": knn_bytes / (knn_ms / 1e3) / 1e9, "call_ms": paths[kpath]["knn_ms"]}
    knn["traffic"] = KNN_DRAM_BYTES_PER_QUERY * Q_KNN
    rad["traffic"] = RADIUS_DRAM_BYTES_PER_QUERY * Q_RADIUS
    dom = knn if knn_ms >= rad_ms else rad
    roofline = {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["achieved"], "peak": peak, "unit": "GB/s",
                "frac": dom["achieved"] / peak, "peak_source": peak_kind, "traffic": dom["traffic"],
                "ms_per_launch": dom["ms"], "call_ms": dom["call_ms"],
                "traffic_source": "DRAM read + write bytes per query of the search kernel from one ncu capture "
                                  "(6M-point tile at the same density, 200k queries), times this step's queries",
                "algorithmic_bytes": "radius 24 + 28 per neighbour; kNN 24 + 36 k per query",
                "other": {"kernel": (rad if dom is knn else knn)["kernel"],
                          "achieved": (rad if dom is knn else knn)["achieved"],
                          "frac": (rad if dom is knn else knn)["achieved"] / peak,
                          "ms_per_launch": (rad if dom is knn else knn)["ms"]}}
    build_bytes = BUILD_BYTES_PER_POINT * N_POINTS + BUILD_BYTES_PER_NODE * info.n_total
    build = {"ms": 1e3 * build_s, "mpts_s": N_POINTS / build_s / 1e6, "gbs": build_bytes / build_s / 1e9,
             "frac": build_bytes / build_s / 1e9 / peak, "nodes": info.n_total, "leaves": info.n_leaf,
             "depth": info.max_depth_seen, "upload_ms": 1e3 * upload_s,
             "sort": "8 passes over the whole keys" if args.sort_8pass else
                     "4 passes over the upper key halves, then the runs of equal upper halves",
             "includes": "bbox + encode + sort + reorder + octree build from points resident in HBM, host syncs "
                         "included (wall clock)"}

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(world, {"search_path": args.search}),
            "radius_qps": chosen["radius_qps"], "knn_qps": chosen["knn_qps"],
            "avg_neighbours": chosen["avg_neighbours"], "paths": paths,
            "batched_vs_plain": (paths["engine"]["qps"] / paths["plain"]["qps"]
                                 if "engine" in paths and "plain" in paths else None),
            # the batched search with FP32 filters (both; the radius filter only) against the plain FP64 path
            "batched_fp32_vs_plain": {k: paths[k]["qps"] / paths["plain"]["qps"]
                                      for k in ("engine_fp32", "engine_fp32_radius") if k in paths and "plain" in paths},
            "engine_config": eng_cfg,
            "build": build, "roofline": roofline, "cpu_baseline": None, "parity": None,
            "batched": None, "serving": None, "large": None,
            "e2e": {"value": e2e_val, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "detail": e2e_detail},
            "gpu_launches": LAUNCHES_PER_STEP[args.search] * args.steps, "clocks": clk,
        }
        _STATE["line"] = line  # from here on the deadline prints what has been measured

    # the reference CPU path on a bounded sample of the same queries, and that sample's results through every
    # GPU search path compared with the reference's (set differences, kNN differences, max d^2 error)
    if rank == 0 and world == 1 and not args.no_cpu:
        res = _section("cpu_baseline", lambda: cpu_leg(args, xyz_h, h, eng, proxy, eng_cfg))
        if "error" in res:
            line["cpu_baseline"] = None
            line["parity"] = res
        else:
            line["cpu_baseline"], line["parity"] = res["cpu"], res["parity"]
    if world == 1 and not args.no_batched:
        line["batched"] = _section("batched", lambda: run_batched(args, dev))
        gc.collect()
        torch.cuda.empty_cache()
    if world == 1 and not args.no_serve:
        line["serving"] = _section("serving", lambda: run_serving(args, dev))
        gc.collect()
        torch.cuda.empty_cache()
    if world == 1 and args.large:
        L.oct_cloud_destroy(h)  # room for the large cloud
        h = None
        eng.close()
        gc.collect()
        torch.cuda.empty_cache()
        L.oct_trim_cloud_memory(dev)  # what earlier sections' clouds left in the cloud pool goes back too
        line["large"] = _section("large", lambda: run_large(args, dev))
    if rank == 0:
        _emit(line)
    if h is not None:
        L.oct_cloud_destroy(h)
    return 0


# ----------------------------------------------------- deadline and sections ---
_STATE = {"line": None, "section": None, "printed": False}
_PRINT_LOCK = threading.Lock()


def _emit(line):
    with _PRINT_LOCK:
        if _STATE["printed"]:
            return
        _STATE["printed"] = True
        print(json.dumps(line), flush=True)


def _start_deadline(seconds: float):
    """After ``seconds`` print the line measured so far (the unfinished section named) and exit; a run whose
    headline is not measured by then exits non-zero."""
    def fire():
        line = _STATE["line"]
        if line is None:
            sys.stderr.write(f"bench: deadline of {seconds:g} s passed in section {_STATE['section']!r} before the "
                             "headline was measured\n")
            sys.stderr.flush()
            os._exit(3)
        line = dict(line)
        line["incomplete"] = {"section": _STATE["section"], "deadline_s": seconds}
        _emit(line)
        os._exit(0)

    t = threading.Timer(seconds, fire)
    t.daemon = True
    t.start()
    return t


def _section(name, fn):
    """Run one auxiliary section; an exception is reported in its place instead of ending the run."""
    _STATE["section"] = name
    t0 = time.perf_counter()
    try:
        out = fn()
    except Exception as exc:  # noqa: BLE001 - reported in the JSON line
        traceback.print_exc()
        out = {"error": f"{type(exc).__name__}: {exc}"}
    if isinstance(out, dict):
        out["section_s"] = round(time.perf_counter() - t0, 2)
    _STATE["section"] = None
    return out


def main():
    global N_POINTS, TILE_M, Q_RADIUS, Q_KNN
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--radius-group", type=int, default=8, help="lanes per query of the plain path")
    ap.add_argument("--knn-bucket", type=int, default=256, help="kNN: subtrees this small are scanned as one range")
    ap.add_argument("--search", default="engine", choices=["plain", "packet", "packet_fp32", "knn_per_query", "engine"],
                    help="search path whose numbers are the headline value")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-cloud batch")
    ap.add_argument("--batched-steps", type=int, default=3, help="timed repetitions of the 256-cloud batch")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving stream")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="length of the serving request stream")
    ap.add_argument("--serve-drain", type=float, default=10.0,
                    help="seconds each server may take after the stream ends before it is stopped")
    ap.add_argument("--serve-slots", type=int, default=3, help="batches the serving scheduler keeps in flight")
    ap.add_argument("--serve-max-batch", type=int, default=512 << 10, help="centres per serving batch at most")
    ap.add_argument("--serve-max-wait", type=float, default=40.0,
                    help="ms after which a queued request is admitted ahead of smaller ones")
    ap.add_argument("--serve-fifo", action="store_true", help="admit serving requests in arrival order only")
    ap.add_argument("--serve-no-graph", action="store_true", help="serving batches launched directly, not as graphs")
    ap.add_argument("--large", action="store_true", help="also run the 500M-point skewed cloud (not in the default run)")
    ap.add_argument("--large-points", type=int, default=500_000_000)
    ap.add_argument("--large-queries", type=int, default=10_000_000)
    ap.add_argument("--large-k", type=int, default=1000)
    ap.add_argument("--points", type=int, default=N_POINTS, help="cloud size (smaller cases for profiling)")
    ap.add_argument("--queries", type=int, default=Q_RADIUS, help="radius and kNN queries per step, each")
    ap.add_argument("--sort-8pass", action="store_true", help="build with the 8-pass sort (the split sort by default)")
    ap.add_argument("--paths", default="", help="comma-separated search paths to time (default: all); the "
                                                 "--search path always runs")
    ap.add_argument("--deadline", type=float, default=1200.0,
                    help="seconds after which the line measured so far is printed (unfinished section named)")
    args = ap.parse_args()
    if args.points != N_POINTS:
        TILE_M = TILE_M * math.sqrt(args.points / N_POINTS)  # same point density
        N_POINTS = args.points
    Q_RADIUS = Q_KNN = args.queries
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.deadline > 0:
        _start_deadline(args.deadline)
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
