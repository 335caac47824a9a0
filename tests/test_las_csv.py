"""LAS files (octrees_benchmark_b200/las.py) and the reference-format benchmark
CSVs (octrees_benchmark_b200/bench_csv.py).

CPU: a LAS 1.2 round trip for point formats 0-3 (coordinates are exactly
X * scale + offset, metadata and header fields as written), a hand-made LAS 1.4
header with the 64-bit point count and extra bytes per record, rejected inputs;
the CSV statistics (upper median, population deviation) and column layouts.
GPU: the driver end to end on a small tile, read back from its files.
"""
import csv
import struct

import numpy as np
import pytest

from octrees_benchmark_b200 import bench_csv
from octrees_benchmark_b200.las import read_header, read_las, write_las
from octrees_benchmark_b200.synth import lidar_tile


@pytest.mark.parametrize("fmt", [0, 1, 2, 3])
def test_las_round_trip(tmp_path, fmt):
    xyz = lidar_tile(5000, 40.0, 3) + np.array([500000.0, 4200000.0, 10.0])
    rng = np.random.default_rng(fmt)
    meta = {"intensity": rng.integers(0, 65535, len(xyz)), "return_number": rng.integers(1, 5, len(xyz)),
            "number_of_returns": rng.integers(1, 7, len(xyz)), "classification": rng.integers(0, 20, len(xyz)),
            "scan_angle_rank": rng.integers(-90, 90, len(xyz)), "user_data": rng.integers(0, 255, len(xyz)),
            "point_source_id": rng.integers(0, 65535, len(xyz)), "scan_direction_flag": rng.integers(0, 2, len(xyz)),
            "edge_of_flight_line": rng.integers(0, 2, len(xyz)), "gps_time": rng.uniform(0, 1e6, len(xyz))}
    path = tmp_path / f"t{fmt}.las"
    stored = write_las(path, xyz, scale=(0.001, 0.001, 0.01), point_format=fmt, metadata=meta)
    got, m = read_las(path, metadata=True)
    assert np.array_equal(got, stored)  # bitwise: the same X * scale + offset
    assert np.abs(got - xyz).max() <= 0.005 + 1e-9
    h = read_header(open(path, "rb").read())
    assert h.version == (1, 2) and h.point_format == fmt and h.n_points == len(xyz)
    assert np.array_equal(h.mins, stored.min(0)) and np.array_equal(h.maxs, stored.max(0))
    for k in ("intensity", "return_number", "number_of_returns", "classification", "user_data", "point_source_id",
              "scan_direction_flag", "edge_of_flight_line"):
        assert np.array_equal(m[k].astype(np.int64), np.asarray(meta[k]).astype(np.int64)), k
    assert np.array_equal(m["scan_angle_rank"].astype(np.int64), meta["scan_angle_rank"])
    if fmt in (1, 3):
        assert np.array_equal(m["gps_time"], meta["gps_time"])


def test_las_14_header_and_extra_bytes(tmp_path):
    # a LAS 1.4 file with format 1, 4 extra bytes per record, the legacy count 0 and the 64-bit count set
    n = 10
    hdr = bytearray(375)
    hdr[0:4] = b"LASF"
    hdr[24], hdr[25] = 1, 4
    struct.pack_into("<HIIBHI", hdr, 94, 375, 375, 0, 1, 32, 0)
    struct.pack_into("<3d", hdr, 131, 0.5, 0.25, 0.125)
    struct.pack_into("<3d", hdr, 155, 100.0, 200.0, 300.0)
    struct.pack_into("<Q", hdr, 247, n)
    rec = bytearray()
    for i in range(n):
        rec += struct.pack("<iiiHBBbBHd", i, -i, 2 * i, 7, 0x09, 2, -3, 4, 5, 1.5 * i) + b"\xaa\xbb\xcc\xdd"
    path = tmp_path / "v14.las"
    path.write_bytes(bytes(hdr) + bytes(rec))
    xyz, m = read_las(path, metadata=True)
    i = np.arange(n, dtype=np.float64)
    assert np.array_equal(xyz, np.stack([i * 0.5 + 100.0, -i * 0.25 + 200.0, 2 * i * 0.125 + 300.0], 1))
    assert (m["return_number"] == 1).all() and (m["number_of_returns"] == 1).all()
    assert np.array_equal(m["gps_time"], 1.5 * i)


def test_las_rejects(tmp_path):
    bad = tmp_path / "bad.las"
    bad.write_bytes(b"NOPE" + bytes(300))
    with pytest.raises(ValueError):
        read_las(bad)
    ok = tmp_path / "ok.las"
    write_las(ok, lidar_tile(100, 10.0, 1))
    buf = bytearray(ok.read_bytes())
    buf[104] = 6  # an extended (1.4) point format
    ok.write_bytes(bytes(buf))
    with pytest.raises(ValueError):
        read_las(ok)
    with pytest.raises(ValueError):
        write_las(tmp_path / "far.las", np.array([[1e9, 0.0, 0.0]]), scale=(1e-3, 1e-3, 1e-3), offset=(0, 0, 0))


def test_csv_stats_and_columns():
    s = bench_csv.Stats([0.4, 0.1, 0.3, 0.2])
    assert s.median() == 0.3  # the upper median, values[size / 2] after sorting
    assert abs(s.stdev() - np.std([0.4, 0.1, 0.3, 0.2])) < 1e-15  # population deviation
    assert abs(s.accumulated() - 1.0) < 1e-15
    row = bench_csv.search_row("2026-01-01-00:00:00", "HilbertEncoder3D", 10, "neighborsPrune_gpu", "sphere", "2.5",
                               4, False, s, 12.5)
    assert len(row.strip().split(",")) == len(bench_csv.SEARCH_HEADER.strip().split(",")) == 21
    assert len(bench_csv.BUILD_HEADER.strip().split(",")) == 20
    assert len(bench_csv.ENCODING_HEADER.strip().split(",")) == 8
    assert bench_csv.fmt(0.000123456789) == "0.000123457" and bench_csv.fmt(True) == "1"


@pytest.mark.gpu
def test_csv_driver_end_to_end(tmp_path):
    las = tmp_path / "tile.las"
    write_las(las, lidar_tile(40_000, 90.0, 9))
    out = tmp_path / "out"
    args = ["--las", str(las), "--kernels", "sphere,cube", "--radii", "1,2.5",
            "--algos", "neighborsPrune,neighbors,neighborsStruct,neighborsApprox", "--approx-tol", "3",
            "--knn", "10,50", "--searches", "500", "--repeats", "2", "--warmup", "--out-dir", str(out)]
    bench_csv.main(args)
    files = sorted(p.name for p in out.iterdir())
    assert len(files) == 3 and any(f.endswith("-build.csv") for f in files) and any(f.endswith("-encoding.csv")
                                                                                 for f in files)
    main = [f for f in files if not f.endswith(("-build.csv", "-encoding.csv"))][0]
    rows = list(csv.DictReader(open(out / main)))
    # 3 exact algorithms x 2 kernels x 2 radii, approx upper + lower x 2 x 2, 2 kNN
    assert len(rows) == 12 + 8 + 2
    byop = {}
    for r in rows:
        assert r["octree"] == "linOct" and r["point_type"] == "PointsAoS" and r["npoints"] == "40000"
        assert r["num_searches"] == "500" and r["repeats"] == "2" and r["openmp_schedule"] == "cuda"
        byop[(r["operation"], r["kernel"], r["radius"])] = float(r["avg_result_size"])
    # every neighbours count the same through each exact algorithm; approx bounds around them
    for kern in ("sphere", "cube"):
        for rad in ("1", "2.5"):
            p = byop[("neighborsPrune_gpu", kern, rad)]
            assert p == byop[("neighbors_gpu", kern, rad)] == byop[("neighborsStruct_gpu", kern, rad)]
            assert byop[("neighborsApproxLower_gpu", kern, rad)] <= p <= byop[("neighborsApproxUpper_gpu", kern, rad)]
    assert byop[("KNNV2_gpu", "kNN", "10")] == 10 and byop[("KNNV2_gpu", "kNN", "50")] == 50
    build = list(csv.DictReader(open(out / [f for f in files if f.endswith("-build.csv")][0])))
    assert len(build) == 1 and int(build[0]["number_of_nodes"]) > 1 and float(build[0]["build_time"]) > 0
