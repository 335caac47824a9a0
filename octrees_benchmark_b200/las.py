"""LAS point-cloud files: a reader and a writer for LAS 1.2 point formats 0-3.

The reference reads LiDAR clouds from LAS files through LASlib
(inc/readers/las_file_reader_parallel.hpp:23-145), which is not available
here; this module reads the same files in numpy.  A point's coordinates are
``X * scale + offset`` per axis in double precision, two roundings in that
order, exactly the reference's ``get_X() * xScale + xOffset``
(las_file_reader_parallel.hpp:66-70), and the metadata fields are the ones
its ``readMeta`` keeps (intensity, return number, number of returns, scan
direction, edge of flight line, classification, scan angle rank, user data,
point source ID; 104-115).  Points come back in file order (the reference
gives point i the id i).

LAS 1.3 and 1.4 files with the legacy point formats 0-3 are read as well
(1.4: the 64-bit point count when the legacy one is 0); formats 4-10
(waveforms, extended records) are rejected with a ValueError.

The writer stores point format 0, 1, 2 or 3 with the given scale and offset
(coordinates rounded to the nearest step), header fields filled as LAS 1.2
asks (bounds, counts by return).
"""
from __future__ import annotations

import datetime
import struct

import numpy as np

_HEADER_12 = 227
# byte layout of the records of point formats 0-3 (LAS 1.2, section 2.6)
_BASE = [("X", "<i4"), ("Y", "<i4"), ("Z", "<i4"), ("intensity", "<u2"), ("flags", "u1"),
         ("classification", "u1"), ("scan_angle_rank", "i1"), ("user_data", "u1"), ("point_source_id", "<u2")]
_FORMATS = {
    0: _BASE,
    1: _BASE + [("gps_time", "<f8")],
    2: _BASE + [("red", "<u2"), ("green", "<u2"), ("blue", "<u2")],
    3: _BASE + [("gps_time", "<f8"), ("red", "<u2"), ("green", "<u2"), ("blue", "<u2")],
}


class LasHeader:
    """The public header block fields this module uses."""

    def __init__(self, version, point_format, record_length, n_points, offset_to_points, scale, offset, mins, maxs):
        self.version = version
        self.point_format = point_format
        self.record_length = record_length
        self.n_points = n_points
        self.offset_to_points = offset_to_points
        self.scale = np.asarray(scale, np.float64)
        self.offset = np.asarray(offset, np.float64)
        self.mins = np.asarray(mins, np.float64)
        self.maxs = np.asarray(maxs, np.float64)


def read_header(buf: bytes) -> LasHeader:
    if len(buf) < _HEADER_12 or buf[:4] != b"LASF":
        raise ValueError("not a LAS file (no LASF signature)")
    vmaj, vmin = buf[24], buf[25]
    offset_to_points, = struct.unpack_from("<I", buf, 96)
    fmt = buf[104] & 0x3F  # the top two bits flag compression (LAZ), not supported
    if buf[104] & 0xC0:
        raise ValueError("compressed (LAZ) point data is not supported")
    rec_len, = struct.unpack_from("<H", buf, 105)
    n, = struct.unpack_from("<I", buf, 107)
    scale = struct.unpack_from("<3d", buf, 131)
    offset = struct.unpack_from("<3d", buf, 155)
    mx, mnx, my, mny, mz, mnz = struct.unpack_from("<6d", buf, 179)
    if (vmaj, vmin) >= (1, 4) and n == 0 and len(buf) >= 255:
        n, = struct.unpack_from("<Q", buf, 247)
    if fmt not in _FORMATS:
        raise ValueError(f"point data format {fmt} is not supported (0-3 are)")
    return LasHeader((vmaj, vmin), fmt, rec_len, n, offset_to_points, scale, offset, (mnx, mny, mnz), (mx, my, mz))


def read_las(path, metadata: bool = False):
    """(xyz float64 (n, 3)[, metadata dict of arrays]) of a LAS file, in file order."""
    with open(path, "rb") as f:
        buf = f.read()
    h = read_header(buf)
    fields = _FORMATS[h.point_format]
    base = np.dtype(fields)
    if h.record_length < base.itemsize:
        raise ValueError(f"point record length {h.record_length} below the {base.itemsize} bytes of format "
                         f"{h.point_format}")
    # records may carry extra bytes after the standard fields
    dt = np.dtype({"names": base.names, "formats": [base.fields[k][0] for k in base.names],
                   "offsets": [base.fields[k][1] for k in base.names], "itemsize": h.record_length})
    end = h.offset_to_points + h.n_points * h.record_length
    if end > len(buf):
        raise ValueError("the file is shorter than its header's point count")
    rec = np.frombuffer(buf, dtype=dt, count=h.n_points, offset=h.offset_to_points)
    xyz = np.empty((h.n_points, 3), np.float64)
    for a, name in enumerate("XYZ"):
        xyz[:, a] = rec[name].astype(np.float64) * h.scale[a] + h.offset[a]
    if not metadata:
        return xyz
    fl = rec["flags"]
    meta = {
        "intensity": rec["intensity"].astype(np.float64),
        "return_number": (fl & 0x07).astype(np.uint16),
        "number_of_returns": ((fl >> 3) & 0x07).astype(np.uint16),
        "scan_direction_flag": ((fl >> 6) & 0x01).astype(np.uint16),
        "edge_of_flight_line": ((fl >> 7) & 0x01).astype(np.uint16),
        "classification": rec["classification"].astype(np.uint16),
        "scan_angle_rank": rec["scan_angle_rank"].astype(np.int8),
        "user_data": rec["user_data"].astype(np.uint16),
        "point_source_id": rec["point_source_id"].astype(np.uint16),
    }
    if "gps_time" in base.names:
        meta["gps_time"] = rec["gps_time"].astype(np.float64)
    return xyz, meta


def write_las(path, xyz, scale=(0.001, 0.001, 0.001), offset=None, point_format: int = 0, metadata=None,
              system_id: str = "octrees_benchmark_b200", software: str = "octrees_benchmark_b200 las.py"):
    """Write points as a LAS 1.2 file.  Coordinates are stored as
    round((x - offset) / scale); ``offset`` defaults to the per-axis minimum
    rounded down to a multiple of the scale.  ``metadata`` (optional) holds
    arrays named like read_las's."""
    if point_format not in _FORMATS:
        raise ValueError("point formats 0-3 only")
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    n = len(xyz)
    scale = np.asarray(scale, np.float64)
    if offset is None:
        offset = np.floor((xyz.min(axis=0) if n else np.zeros(3)) / scale) * scale
    offset = np.asarray(offset, np.float64)
    q = np.rint((xyz - offset) / scale)
    if n and (q.min() < -2**31 or q.max() > 2**31 - 1):
        raise ValueError("coordinates do not fit 32-bit integers at this scale and offset")
    dt = np.dtype(_FORMATS[point_format])
    rec = np.zeros(n, dt)
    rec["X"], rec["Y"], rec["Z"] = q[:, 0], q[:, 1], q[:, 2]
    meta = metadata or {}
    rn = np.asarray(meta.get("return_number", np.ones(n)), np.uint8) & 7
    nr = np.asarray(meta.get("number_of_returns", np.ones(n)), np.uint8) & 7
    sd = np.asarray(meta.get("scan_direction_flag", np.zeros(n)), np.uint8) & 1
    ed = np.asarray(meta.get("edge_of_flight_line", np.zeros(n)), np.uint8) & 1
    rec["flags"] = rn | (nr << 3) | (sd << 6) | (ed << 7)
    for name in ("intensity", "classification", "scan_angle_rank", "user_data", "point_source_id", "gps_time"):
        if name in meta and name in dt.names:
            rec[name] = meta[name]
    stored = rec[["X", "Y", "Z"]]
    back = np.stack([stored[a].astype(np.float64) * scale[i] + offset[i] for i, a in enumerate("XYZ")], 1) \
        if n else np.zeros((0, 3))
    mins = back.min(axis=0) if n else np.zeros(3)
    maxs = back.max(axis=0) if n else np.zeros(3)
    by_return = [int(np.count_nonzero(rn == r)) for r in range(1, 6)]
    today = datetime.date.today()
    hdr = bytearray(_HEADER_12)
    hdr[0:4] = b"LASF"
    hdr[24], hdr[25] = 1, 2
    hdr[26:58] = system_id.encode()[:32].ljust(32, b"\0")
    hdr[58:90] = software.encode()[:32].ljust(32, b"\0")
    struct.pack_into("<HH", hdr, 90, today.timetuple().tm_yday, today.year)
    struct.pack_into("<HIIBHI", hdr, 94, _HEADER_12, _HEADER_12, 0, point_format, dt.itemsize, n)
    struct.pack_into("<5I", hdr, 111, *by_return)
    struct.pack_into("<3d", hdr, 131, *scale)
    struct.pack_into("<3d", hdr, 155, *offset)
    struct.pack_into("<6d", hdr, 179, maxs[0], mins[0], maxs[1], mins[1], maxs[2], mins[2])
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(rec.tobytes())
    return back
