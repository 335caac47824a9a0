"""Benchmark driver with the reference's CSV output, so that its plotting
scripts read GPU results beside CPU ones.

    python -m octrees_benchmark_b200.bench_csv [--las FILE | --points N --tile M --seed S]
        [--encoder hilbert] [--leaf 64] [--kernels sphere,cube] [--radii 1,2.5,5]
        [--algos neighborsPrune,neighbors,neighborsStruct,neighborsApprox] [--approx-tol 50]
        [--knn 10,50] [--searches 10000 | --sequential] [--repeats 5] [--warmup]
        [--out-dir DIR] [--comment gpu]

Files and columns follow the reference (inc/benchmarking/neighbor_benchmarks.hpp:
119-171, build_log.hpp:75-120, encoding_log.hpp:33-53, src/main.cpp:305-339):
``<input>-<date>.csv`` with one row per (operation, kernel, radius or k):
date, octree, point_type, encoder, npoints, operation, kernel, radius,
num_searches, sequential_searches, repeats, accumulated, mean, median, stdev,
used_warmup, warmup_time, avg_result_size, tolerance_percentage,
openmp_threads, openmp_schedule; ``<input>-<date>-build.csv`` and
``<input>-<date>-encoding.csv`` with the build and encoding logs.  Times are
seconds per repetition, each repetition answering all searches (the
reference's OpenMP loop over the search set is one batched call here, timed on
the host around the call with its copies in and out); median is the upper
median and stdev the population deviation, as the reference computes them.
The device rows carry openmp_threads = 0 and openmp_schedule = "cuda", and the
operation name gets the ``--comment`` suffix the reference appends
(``neighborsPrune_gpu``).  Search centres are cloud points chosen as the
reference's SearchSet does (random indices, or every point in order with
--sequential; the random generator differs).
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os
import statistics
import time

import numpy as np

from . import LinearOctree
from .capi import OctTreeInfo, check
from .synth import lidar_tile, query_indices

SEARCH_HEADER = ("date,octree,point_type,encoder,npoints,operation,kernel,radius,num_searches,sequential_searches,"
                 "repeats,accumulated,mean,median,stdev,used_warmup,warmup_time,avg_result_size,tolerance_percentage,"
                 "openmp_threads,openmp_schedule\n")
BUILD_HEADER = ("container,structure,max_leaf_points,enc_type,cloud_size,linear_octree_leaf_time,"
                "linear_octree_internal_time,build_time,memory_used,number_of_nodes,leaf_nodes,internal_nodes,"
                "max_depth_seen,min_radii_seen,repeats,min_warmup_time,l1d_miss,l2d_miss,l3_miss,num_threads\n")
ENCODING_HEADER = "container,enc_type,cloud_size,bbox_time,enc_time,sort_time,repeats,used_warmup\n"
ENCODER_NAMES = {"morton": ("MortonEncoder3D", "mort"), "hilbert": ("HilbertEncoder3D", "hilb")}


def current_date() -> str:
    """getCurrentDate (inc/util.hpp:187-193): %Y-%m-%d-%H:%M:%S, local time."""
    return time.strftime("%Y-%m-%d-%H:%M:%S")


class Stats:
    """BenchmarkingStats (inc/benchmarking/benchmarking_stats.hpp): values in seconds."""

    def __init__(self, values, used_warmup=False, warmup_value=0.0):
        self.values = list(values) or [0.0]
        self.used_warmup = used_warmup
        self.warmup_value = warmup_value

    def accumulated(self):
        return math.fsum(self.values)

    def mean(self):
        return statistics.fmean(self.values)

    def median(self):
        return sorted(self.values)[len(self.values) // 2]

    def stdev(self):
        m = self.mean()
        return math.sqrt(math.fsum((v - m) ** 2 for v in self.values) / len(self.values))


def fmt(v) -> str:
    """A number as C++ stream output prints it (6 significant digits, %g)."""
    if isinstance(v, (bool, np.bool_)):
        return "1" if v else "0"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return f"{float(v):g}"


def search_row(date, encoder_name, npoints, operation, kernel, radius, num_searches, sequential, stats,
               avg_result_size, tolerance=0.0):
    cells = [date, "linOct", "PointsAoS", encoder_name, npoints, operation, kernel, radius, num_searches,
             "sequential" if sequential else "random", len(stats.values), stats.accumulated(), stats.mean(),
             stats.median(), stats.stdev(), stats.used_warmup, stats.warmup_value, avg_result_size, tolerance, 0,
             "cuda"]
    return ",".join(c if isinstance(c, str) else fmt(c) for c in cells) + "\n"


def append(path, header, rows):
    new = not os.path.exists(path) or os.path.getsize(path) == 0
    with open(path, "a") as f:
        if new:
            f.write(header)
        f.writelines(rows)


def timed(fn, repeats, warmup):
    if warmup:
        fn()
    times, last = [], None
    for _ in range(repeats):
        t = time.perf_counter()
        last = fn()
        times.append(time.perf_counter() - t)
    return times, last


def run(args):
    if args.las:
        from .las import read_las
        xyz = read_las(args.las)
        name = os.path.splitext(os.path.basename(args.las))[0]
    else:
        xyz = lidar_tile(args.points, args.tile, args.seed)
        name = f"synthetic_{args.points}"
    os.makedirs(args.out_dir, exist_ok=True)
    date = current_date()
    enc_name, enc_short = ENCODER_NAMES[args.encoder]
    n = len(xyz)
    suffix = f"_{args.comment}" if args.comment else ""

    # encoding + build logs.  The device sorts in one call (oct_encode_sort: upload of the host
    # points, bbox, encode, sort, reorder) and builds in one (oct_build), so sort_time holds the
    # whole sortPoints and build_time the whole construction; the split columns stay 0.
    oc = LinearOctree(xyz, encoder=args.encoder, max_points_leaf=args.leaf)  # first call sizes the buffers
    L, h = oc._L, oc.handle
    pts = np.ascontiguousarray(xyz, np.float64)
    box = np.zeros(12)
    info = OctTreeInfo()
    enc_t, build_t = [], []
    for _ in range(args.repeats):
        t0 = time.perf_counter()
        check(L.oct_set_points(h, pts.ctypes.data, n, 0), h, "oct_set_points")
        check(L.oct_encode_sort(h, box.ctypes.data, None, None, None, 0), h, "oct_encode_sort")
        t1 = time.perf_counter()
        check(L.oct_build(h, C.byref(info)), h, "oct_build")
        build_t.append(time.perf_counter() - t1)
        enc_t.append(t1 - t0)
    mem = C.c_uint64(0)
    check(L.oct_cloud_memory(h, C.byref(mem)), h, "oct_cloud_memory")
    min_radius = float(min(oc.export()["radii"][oc.max_depth_seen]))
    append(os.path.join(args.out_dir, f"{name}-{date}-encoding.csv"), ENCODING_HEADER,
           [f"PointsAoS,{enc_short},{n},0,0,{fmt(statistics.fmean(enc_t))},{args.repeats},{fmt(args.warmup)}\n"])
    append(os.path.join(args.out_dir, f"{name}-{date}-build.csv"), BUILD_HEADER,
           [f"PointsAoS,linOct,{args.leaf},{enc_short},{n},0,0,{fmt(statistics.fmean(build_t))},{mem.value},"
            f"{oc.n_total},{oc.n_leaf},{oc.n_internal},{oc.max_depth_seen},{fmt(min_radius)},{args.repeats},0,0,0,0,"
            "0\n"])

    # the search set: cloud points (SearchSet, search_set.hpp:25-36), in the sorted cloud's indexing
    _, _, sxyz = oc.sorted_points()
    if args.sequential:
        centres = sxyz
    else:
        centres = sxyz[query_indices(min(args.searches, n), n, seed=42)]
    ns = len(centres)
    rows = []
    for algo in args.algos:
        for kernel in args.kernels:
            for r in args.radii:
                if algo == "neighborsApprox":
                    for tol in args.approx_tol:
                        for upper in (True, False):
                            times, res = timed(lambda: oc.neighborsApprox(centres, r, tol, upper, kernel),
                                               args.repeats, args.warmup)
                            op = f"neighborsApprox{'Upper' if upper else 'Lower'}{suffix}"
                            rows.append(search_row(date, enc_name, n, op, kernel, fmt(r), ns, args.sequential,
                                                   Stats(times, args.warmup), float(np.mean(res[2])) if ns else 0,
                                                   tol))
                    continue
                if algo == "neighborsStruct":
                    times, res = timed(lambda: oc.neighborsStruct(centres, r, kernel), args.repeats, args.warmup)
                    avg = float(np.mean(res[2])) if ns else 0.0
                else:
                    times, res = timed(lambda: oc.radius_search(centres, r, kernel, algo), args.repeats, args.warmup)
                    avg = float(res[0][-1]) / ns if ns else 0.0
                rows.append(search_row(date, enc_name, n, algo + suffix, kernel, fmt(r), ns, args.sequential,
                                       Stats(times, args.warmup), avg))
    for k in args.knn:
        times, res = timed(lambda: oc.knn(centres, k), args.repeats, args.warmup)
        rows.append(search_row(date, enc_name, n, "KNNV2" + suffix, "kNN", str(k), ns, args.sequential,
                               Stats(times, args.warmup), float(np.mean(res[2])) if ns else 0.0))
    path = os.path.join(args.out_dir, f"{name}-{date}.csv")
    append(path, SEARCH_HEADER, rows)
    oc.close()
    return path


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--las", help="LAS file (point formats 0-3); default: a synthetic tile")
    ap.add_argument("--points", type=int, default=1_000_000)
    ap.add_argument("--tile", type=float, default=500.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--encoder", choices=sorted(ENCODER_NAMES), default="hilbert")
    ap.add_argument("--leaf", type=int, default=128)
    ap.add_argument("--kernels", type=lambda s: s.split(","), default=["sphere"])
    ap.add_argument("--radii", type=lambda s: [float(v) for v in s.split(",")], default=[2.5])
    ap.add_argument("--algos", type=lambda s: s.split(","), default=["neighborsPrune"])
    ap.add_argument("--approx-tol", type=lambda s: [float(v) for v in s.split(",")], default=[50.0],
                    help="neighborsApprox tolerance percentages (used as the precision level, as the reference does)")
    ap.add_argument("--knn", type=lambda s: [int(v) for v in s.split(",") if v], default=[])
    ap.add_argument("--searches", type=int, default=10_000)
    ap.add_argument("--sequential", action="store_true", help="search every point in order")
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--warmup", action="store_true")
    ap.add_argument("--out-dir", default="out")
    ap.add_argument("--comment", default="gpu", help="suffix of the operation names")
    args = ap.parse_args(argv)
    print(run(args))


if __name__ == "__main__":
    main()
