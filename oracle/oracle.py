"""Test infrastructure: ctypes front ends for the two CPU checkers.

* ``Port`` loads oracle/_build/liboctree_oracle.so, the plain-C restatement of
  the reference algorithm (octree_oracle.c).
* ``Reference`` loads oracle/_ref/libref_octree.so, the UNMODIFIED reference
  headers compiled by ``make -C oracle ref REFERENCE=<dir>`` behind a thin C bridge
  (ref_bridge.cpp).  It exists wherever it was built (it is git-ignored but
  travels with the working tree); ``reference_available()`` says whether it is.

Only tests/, tests/golden/make_golden.py and bench.py's CPU-baseline leg import
this module.  The product never does.

Conventions: encoder 1 Morton / 5 Hilbert; kernel 0 circle, 1 sphere, 2 square,
3 cube; algo 1 neighbors, 2 neighborsPrune, 3 neighborsStruct; ``box`` is the
12-vector (center, radii, min, max); clouds are (n, 3) float64 arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liboctree_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_octree.so")

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build_port() -> str:
    """Compile the C restatement (cheap; gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return PORT_SO


def build_reference(reference_dir: str | None = None) -> str | None:
    """Compile the reference bridge from the reference checkout ``reference_dir``
    (else $OCTREE_REFERENCE_DIR).  Without one, keeps a prebuilt library."""
    ref = reference_dir or os.environ.get("OCTREE_REFERENCE_DIR")
    if not ref or not os.path.isdir(os.path.join(ref, "inc")):
        return REF_SO if os.path.exists(REF_SO) else None
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={ref}"], check=True)
    return REF_SO


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Port:
    """The plain-C restatement of the reference algorithm."""

    _lib = None

    def __init__(self):
        if Port._lib is None:
            if not os.path.exists(PORT_SO):
                build_port()
            L = C.CDLL(PORT_SO)
            L.orc_bbox.argtypes = [_f64p, C.c_uint64, _f64p]
            L.orc_anchor.argtypes = [C.c_double] * 3
            L.orc_anchor.restype = C.c_uint64
            for nm in ("orc_morton_encode", "orc_hilbert_encode"):
                getattr(L, nm).argtypes = [C.c_uint64] * 3
                getattr(L, nm).restype = C.c_uint64
            for nm in ("orc_morton_decode", "orc_hilbert_decode"):
                getattr(L, nm).argtypes = [C.c_uint64] + [C.POINTER(C.c_uint64)] * 3
            L.orc_encode.argtypes = [C.c_int, _f64p, C.c_uint64, _f64p, _u64p]
            L.orc_sort.argtypes = [_u64p, C.c_uint64, _u32p]
            L.orc_build.argtypes = [C.c_int, _u64p, C.c_uint64, C.c_uint64, _f64p]
            L.orc_build.restype = C.c_void_p
            L.orc_tree_info.argtypes = [C.c_void_p, _u64p]
            L.orc_tree_arrays.argtypes = [C.c_void_p, _u32p, _u64p, _f64p, _f64p, _f64p]
            L.orc_tree_free.argtypes = [C.c_void_p]
            L.orc_radius_count.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, _f64p, C.c_uint64, _f64p, _u64p]
            L.orc_radius_fill.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, _f64p, C.c_uint64, _f64p, _u64p,
                                          _u64p]
            L.orc_struct_ranges_count.argtypes = [C.c_void_p, _f64p, C.c_int, _f64p, C.c_uint64, _f64p, _u64p]
            L.orc_struct_ranges_fill.argtypes = [C.c_void_p, _f64p, C.c_int, _f64p, C.c_uint64, _f64p, _u64p,
                                                 _u64p]
            L.orc_approx_ranges_count.argtypes = [C.c_void_p, _f64p, C.c_int, _f64p, C.c_uint64, _f64p, C.c_uint32,
                                                  C.c_int, _u64p]
            L.orc_approx_ranges_fill.argtypes = [C.c_void_p, _f64p, C.c_int, _f64p, C.c_uint64, _f64p, C.c_uint32,
                                                 C.c_int, _u64p, _u64p]
            L.orc_knn.argtypes = [C.c_void_p, _f64p, C.c_uint64, _f64p, C.c_uint64, C.c_uint64, _u64p, _f64p,
                                  _u64p]
            Port._lib = L
        self.L = Port._lib

    # -- encoding ---------------------------------------------------------
    def bbox(self, xyz):
        xyz = _f64(xyz)
        box = np.zeros(12)
        self.L.orc_bbox(xyz, len(xyz), box)
        return box

    def anchor(self, p, c, r):
        return int(self.L.orc_anchor(p, c, r))

    def encode_xyz(self, encoder, x, y, z):
        fn = self.L.orc_hilbert_encode if encoder == 5 else self.L.orc_morton_encode
        return int(fn(x, y, z))

    def decode_key(self, encoder, key):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        fn = self.L.orc_hilbert_decode if encoder == 5 else self.L.orc_morton_decode
        fn(key, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def encode(self, encoder, xyz, box):
        xyz = _f64(xyz)
        keys = np.zeros(len(xyz), np.uint64)
        self.L.orc_encode(encoder, xyz, len(xyz), _f64(box), keys)
        return keys

    def sort(self, keys):
        keys = np.array(keys, dtype=np.uint64, copy=True)
        perm = np.zeros(len(keys), np.uint32)
        self.L.orc_sort(keys, len(keys), perm)
        return keys, perm

    def encode_sort(self, encoder, xyz):
        """PointEncoder::sortPoints: returns (sorted keys, perm, box, sorted xyz)."""
        xyz = _f64(xyz)
        box = self.bbox(xyz)
        keys, perm = self.sort(self.encode(encoder, xyz, box))
        return keys, perm, box, xyz[perm.astype(np.int64)]

    def build(self, encoder, keys, max_leaf, box):
        return PortTree(self, encoder, keys, max_leaf, box)


class PortTree:
    def __init__(self, port, encoder, keys, max_leaf, box):
        self.port = port
        self.L = port.L
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        self.n = len(keys)
        self.h = self.L.orc_build(encoder, keys, len(keys), max_leaf, _f64(box))
        info = np.zeros(5, np.uint64)
        self.L.orc_tree_info(self.h, info)
        self.n_leaf, self.n_internal, self.n_total, self.max_depth = (int(v) for v in info[1:5])

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_tree_free(self.h)
            self.h = None

    def arrays(self):
        nt = self.n_total
        off = np.zeros(nt + 1, np.uint32)
        rng = np.zeros(2 * nt, np.uint64)
        ctr = np.zeros(3 * nt, np.float64)
        rad = np.zeros(66, np.float64)
        half = np.zeros(3, np.float64)
        self.L.orc_tree_arrays(self.h, off, rng, ctr, rad, half)
        return dict(offsets=off, ranges=rng.reshape(nt, 2), centers=ctr.reshape(nt, 3),
                    radii=rad.reshape(22, 3), half=half)

    def radius(self, xyz, kernel, algo, centers, radii):
        """CSR (offsets uint64[nq+1], indices uint64) in the reference's emission order."""
        xyz, centers = _f64(xyz), _f64(centers)
        nq = len(centers)
        radii = _f64(np.broadcast_to(np.asarray(radii, np.float64), (nq,)))
        counts = np.zeros(nq, np.uint64)
        self.L.orc_radius_count(self.h, xyz, kernel, algo, centers, nq, radii, counts)
        offs = np.zeros(nq + 1, np.uint64)
        np.cumsum(counts, out=offs[1:])
        idx = np.zeros(int(offs[-1]), np.uint64)
        self.L.orc_radius_fill(self.h, xyz, kernel, algo, centers, nq, radii, offs, idx)
        return offs, idx

    def struct_ranges(self, xyz, kernel, centers, radii):
        """neighborsStruct ranges: offsets uint64[nq+1], pairs uint64[m, 2]."""
        xyz, centers = _f64(xyz), _f64(centers)
        nq = len(centers)
        radii = _f64(np.broadcast_to(np.asarray(radii, np.float64), (nq,)))
        counts = np.zeros(nq, np.uint64)
        self.L.orc_struct_ranges_count(self.h, xyz, kernel, centers, nq, radii, counts)
        offs = np.zeros(nq + 1, np.uint64)
        np.cumsum(counts, out=offs[1:])
        pairs = np.zeros(2 * int(offs[-1]), np.uint64)
        self.L.orc_struct_ranges_fill(self.h, xyz, kernel, centers, nq, radii, offs, pairs)
        return offs, pairs.reshape(-1, 2)

    def approx_ranges(self, xyz, kernel, centers, radii, level, upper):
        """neighborsApprox ranges (the traversal cut below depth `level`; `upper`: cut octants added)."""
        xyz, centers = _f64(xyz), _f64(centers)
        nq = len(centers)
        radii = _f64(np.broadcast_to(np.asarray(radii, np.float64), (nq,)))
        counts = np.zeros(nq, np.uint64)
        self.L.orc_approx_ranges_count(self.h, xyz, kernel, centers, nq, radii, int(level), int(bool(upper)), counts)
        offs = np.zeros(nq + 1, np.uint64)
        np.cumsum(counts, out=offs[1:])
        pairs = np.zeros(2 * int(offs[-1]), np.uint64)
        self.L.orc_approx_ranges_fill(self.h, xyz, kernel, centers, nq, radii, int(level), int(bool(upper)), offs,
                                      pairs)
        return offs, pairs.reshape(-1, 2)

    def knn(self, xyz, centers, k):
        xyz, centers = _f64(xyz), _f64(centers)
        nq = len(centers)
        idx = np.zeros(nq * k, np.uint64)
        d2 = np.zeros(nq * k, np.float64)
        cnt = np.zeros(nq, np.uint64)
        self.L.orc_knn(self.h, xyz, len(xyz), centers, nq, k, idx, d2, cnt)
        return idx.reshape(nq, k), d2.reshape(nq, k), cnt


class Reference:
    """The compiled reference implementation (one built cloud per instance)."""

    _lib = None

    @staticmethod
    def lib():
        if Reference._lib is None:
            if not os.path.exists(REF_SO):
                raise RuntimeError("oracle/_ref/libref_octree.so is not built (make -C oracle ref REFERENCE=<dir>)")
            L = C.CDLL(REF_SO)
            L.refo_build.argtypes = [C.c_int, _f64p, C.c_uint64, C.c_uint64, C.c_int]
            L.refo_build.restype = C.c_void_p
            L.refo_free.argtypes = [C.c_void_p]
            L.refo_info.argtypes = [C.c_void_p, _u64p]
            L.refo_times.argtypes = [C.c_void_p, _f64p]
            L.refo_box.argtypes = [C.c_void_p, _f64p]
            L.refo_points.argtypes = [C.c_void_p, _f64p, _u64p, _u64p]
            L.refo_tree.argtypes = [C.c_void_p, _u32p, _u64p, _f64p, _f64p, _f64p]
            L.refo_radius.argtypes = [C.c_void_p, C.c_int, C.c_int, _f64p, C.c_uint64, _f64p, C.c_int]
            L.refo_radius.restype = C.c_uint64
            L.refo_radius_fetch.argtypes = [C.c_void_p, _u64p, _u64p]
            L.refo_struct_range_total.argtypes = [C.c_void_p]
            L.refo_struct_range_total.restype = C.c_uint64
            L.refo_struct_ranges_fetch.argtypes = [C.c_void_p, _u64p, _u64p]
            L.refo_approx.argtypes = [C.c_void_p, C.c_int, _f64p, C.c_uint64, _f64p, C.c_double, C.c_int, C.c_int]
            L.refo_approx.restype = C.c_uint64
            L.refo_knn.argtypes = [C.c_void_p, _f64p, C.c_uint64, C.c_uint64, _u64p, _f64p, _u64p, C.c_int]
            L.refo_time_radius.argtypes = [C.c_void_p, C.c_int, C.c_int, _f64p, C.c_uint64, C.c_double, C.c_int,
                                           C.POINTER(C.c_uint64)]
            L.refo_time_radius.restype = C.c_double
            L.refo_time_knn.argtypes = [C.c_void_p, _f64p, C.c_uint64, C.c_uint64, C.c_int,
                                        C.POINTER(C.c_double)]
            L.refo_time_knn.restype = C.c_double
            L.refo_radius_hash.argtypes = [C.c_void_p, C.c_int, C.c_int, _f64p, C.c_uint64, C.c_double, C.c_int,
                                           _u64p, _u64p]
            L.refo_search_set.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_uint64, _u64p]
            L.refo_radius_axes.argtypes = [C.c_void_p, C.c_int, C.c_int, _f64p, C.c_uint64, _f64p, C.c_int]
            L.refo_radius_axes.restype = C.c_uint64
            L.refo_max_threads.restype = C.c_int
            L.refo_anchor.argtypes = [C.c_double] * 3
            L.refo_anchor.restype = C.c_uint64
            L.refo_encode.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64]
            L.refo_encode.restype = C.c_uint64
            L.refo_decode.argtypes = [C.c_int, C.c_uint64, _u64p]
            Reference._lib = L
        return Reference._lib

    def __init__(self, encoder, xyz, max_leaf, threads=0):
        self.L = Reference.lib()
        xyz = _f64(xyz)
        self.h = self.L.refo_build(encoder, xyz.reshape(-1), len(xyz), max_leaf, threads)
        info = np.zeros(5, np.uint64)
        self.L.refo_info(self.h, info)
        self.n, self.n_leaf, self.n_internal, self.n_total, self.max_depth = (int(v) for v in info)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.refo_free(self.h)
            self.h = None

    def times(self):
        t = np.zeros(5)
        self.L.refo_times(self.h, t)
        return dict(sort=t[0], build=t[1], bbox=t[2], encode=t[3], radix=t[4])

    def box(self):
        b = np.zeros(12)
        self.L.refo_box(self.h, b)
        return b

    def points(self):
        xyz = np.zeros(3 * self.n)
        ids = np.zeros(self.n, np.uint64)
        keys = np.zeros(self.n, np.uint64)
        self.L.refo_points(self.h, xyz, ids, keys)
        return xyz.reshape(self.n, 3), ids, keys

    def arrays(self):
        nt = self.n_total
        off = np.zeros(nt + 1, np.uint32)
        rng = np.zeros(2 * nt, np.uint64)
        ctr = np.zeros(3 * nt, np.float64)
        rad = np.zeros(66, np.float64)
        half = np.zeros(3, np.float64)
        self.L.refo_tree(self.h, off, rng, ctr, rad, half)
        return dict(offsets=off, ranges=rng.reshape(nt, 2), centers=ctr.reshape(nt, 3),
                    radii=rad.reshape(22, 3), half=half)

    def radius(self, kernel, algo, centers, radii, threads=0):
        centers = _f64(centers)
        nq = len(centers)
        radii = _f64(np.broadcast_to(np.asarray(radii, np.float64), (nq,)))
        total = self.L.refo_radius(self.h, kernel, algo, centers.reshape(-1), nq, radii, threads)
        offs = np.zeros(nq + 1, np.uint64)
        idx = np.zeros(int(total), np.uint64)
        self.L.refo_radius_fetch(self.h, offs, idx)
        return offs, idx

    def radius_axes(self, kernel, algo, centers, radii_xyz, threads=0):
        """The Vector-radii overloads (square 2 / cube 3): CSR of indices in the reference's emission order,
        and for algo 3 the ranges as well: (offs, idx, range_offs, pairs)."""
        centers = _f64(centers)
        nq = len(centers)
        r3 = _f64(np.broadcast_to(np.asarray(radii_xyz, np.float64), (nq, 3)))
        total = self.L.refo_radius_axes(self.h, kernel, algo, centers.reshape(-1), nq, r3.reshape(-1), threads)
        offs = np.zeros(nq + 1, np.uint64)
        idx = np.zeros(int(total), np.uint64)
        self.L.refo_radius_fetch(self.h, offs, idx)
        m = self.L.refo_struct_range_total(self.h)
        ro = np.zeros(nq + 1, np.uint64)
        pairs = np.zeros(2 * int(m), np.uint64)
        self.L.refo_struct_ranges_fetch(self.h, ro, pairs)
        return offs, idx, ro, pairs.reshape(-1, 2)

    def struct_ranges(self, kernel, centers, radii, threads=0):
        """ranges of neighborsStruct in the reference's emission order"""
        self.radius(kernel, 3, centers, radii, threads)
        m = self.L.refo_struct_range_total(self.h)
        offs = np.zeros(len(centers) + 1, np.uint64)
        pairs = np.zeros(2 * int(m), np.uint64)
        self.L.refo_struct_ranges_fetch(self.h, offs, pairs)
        return offs, pairs.reshape(-1, 2)

    def approx_ranges(self, kernel, centers, radii, tolerance, upper, threads=0):
        """ranges of neighborsApprox(p, r, tolerancePercentage, upperBound), in the reference's
        emission order (its overloads pass the percentage on as the precision level)"""
        centers = _f64(centers)
        nq = len(centers)
        radii = _f64(np.broadcast_to(np.asarray(radii, np.float64), (nq,)))
        self.L.refo_approx(self.h, kernel, centers.reshape(-1), nq, radii, float(tolerance), int(bool(upper)), threads)
        m = self.L.refo_struct_range_total(self.h)
        offs = np.zeros(nq + 1, np.uint64)
        pairs = np.zeros(2 * int(m), np.uint64)
        self.L.refo_struct_ranges_fetch(self.h, offs, pairs)
        return offs, pairs.reshape(-1, 2)

    def knn(self, centers, k, threads=0):
        centers = _f64(centers)
        nq = len(centers)
        idx = np.zeros(nq * k, np.uint64)
        d2 = np.zeros(nq * k, np.float64)
        cnt = np.zeros(nq, np.uint64)
        self.L.refo_knn(self.h, centers.reshape(-1), nq, k, idx, d2, cnt, threads)
        return idx.reshape(nq, k), d2.reshape(nq, k), cnt

    def radius_hash(self, kernel, algo, centers, radius, threads=0):
        """Per-query neighbour counts and order-independent set hashes (sum of splitmix64(index) mod 2^64)."""
        centers = _f64(centers)
        nq = len(centers)
        counts = np.zeros(nq, np.uint64)
        hashes = np.zeros(nq, np.uint64)
        self.L.refo_radius_hash(self.h, kernel, algo, centers.reshape(-1), nq, float(radius), threads, counts, hashes)
        return counts, hashes

    def time_radius(self, kernel, algo, centers, radius, threads=0):
        tot = C.c_uint64()
        centers = _f64(centers)
        s = self.L.refo_time_radius(self.h, kernel, algo, centers.reshape(-1), len(centers), radius, threads,
                                    C.byref(tot))
        return s, tot.value

    def time_knn(self, centers, k, threads=0):
        chk = C.c_double()
        centers = _f64(centers)
        s = self.L.refo_time_knn(self.h, centers.reshape(-1), len(centers), k, threads, C.byref(chk))
        return s, chk.value

    @staticmethod
    def anchor(p, c, r):
        return int(Reference.lib().refo_anchor(p, c, r))

    @staticmethod
    def encode_xyz(encoder, x, y, z):
        return int(Reference.lib().refo_encode(encoder, x, y, z))

    @staticmethod
    def decode_key(encoder, key):
        out = np.zeros(3, np.uint64)
        Reference.lib().refo_decode(encoder, key, out)
        return tuple(int(v) for v in out)

    @staticmethod
    def search_set(n, cloud_size, sequential=False, all_points=False, repeats=1):
        """The reference's SearchSet indices, (repeats, n) (n = cloud_size with all_points)."""
        m = cloud_size if all_points else n
        out = np.zeros(repeats * m, np.uint64)
        Reference.lib().refo_search_set(n, cloud_size, int(bool(sequential)), int(bool(all_points)), repeats, out)
        return out.reshape(repeats, m)

    @staticmethod
    def max_threads():
        return int(Reference.lib().refo_max_threads())
