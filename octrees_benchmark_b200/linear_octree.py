"""Python front end over the C ABI, with the reference's names.

``LinearOctree(points, encoder, max_points_leaf)`` does what the reference's
``PointEncoder::sortPoints`` (inc/encoding/point_encoder.hpp:484-503) followed by
the ``LinearOctree<Container>`` constructor (inc/structures/linear_octree.hpp:
614-623) do, on the GPU; the search methods are batched forms of
``neighbors`` / ``neighborsPrune`` / ``neighborsStruct`` / ``knn``
(linear_octree.hpp:695-942, 1038-1087): they take an (nq, 3) array of centres
instead of one ``Point``.  As in the reference, the default kernel of the
scalar-radius overloads is ``square``.

Host (numpy) inputs go through the host-buffer form of the ABI; CUDA torch
tensors go through the device-buffer form (``OCT_MEM_DEVICE``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import ALGOS, ENCODERS, KERNELS, OCT_MEM_DEVICE, OctParams, OctSearchConfig, OctTreeInfo, check, lib


def _ptr(a) -> int:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _is_device(a) -> bool:
    return not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


def _sync_current_stream():
    """Wait for the caller's current torch stream: the library reads device
    tensors on its own (non-blocking) streams."""
    import torch

    torch.cuda.current_stream().synchronize()


def _host_f64(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape_last is not None and a.ndim == 1:
        a = a.reshape(-1, shape_last)
    return a


class LinearOctree:
    """A device-resident cloud, SFC-sorted, with its linear octree built."""

    def __init__(self, points, encoder="hilbert", max_points_leaf: int = 128, device: int = 0,
                 radius_group: int = 8, stream=None, packet: bool = True, fp32_filter: bool = False,
                 knn_packet: bool = True, knn_bucket: int = 256, sort_8pass: bool = False):
        self._open(encoder, max_points_leaf, device, radius_group, stream, packet, fp32_filter, knn_packet,
                   knn_bucket, capi.OCT_CLOUD_SORT_8PASS if sort_8pass else 0)
        L, h = self._L, self._h
        dev = _is_device(points)
        if not dev:
            points = _host_f64(points, 3)
        else:
            _sync_current_stream()  # the cloud reads the tensor on its own stream
        self.n = int(points.shape[0])
        check(L.oct_set_points(h, _ptr(points), self.n, OCT_MEM_DEVICE if dev else 0), h, "oct_set_points")
        box = np.zeros(12)
        check(L.oct_encode_sort(h, box.ctypes.data, None, None, None, 0), h, "oct_encode_sort")
        self.box = box
        info = OctTreeInfo()
        check(L.oct_build(h, C.byref(info)), h, "oct_build")
        self.n_leaf = info.n_leaf
        self.n_internal = info.n_internal
        self.n_total = info.n_total
        self.max_depth_seen = info.max_depth_seen

    def _open(self, encoder, max_points_leaf, device, radius_group, stream, packet, fp32_filter, knn_packet,
              knn_bucket, flags=0):
        L = lib()
        self._L = L
        self.encoder = ENCODERS[encoder] if not isinstance(encoder, (int, np.integer)) else int(encoder)
        self.max_points_leaf = int(max_points_leaf)
        p = OctParams(self.max_points_leaf, self.encoder, device, flags)
        h = C.c_void_p()
        st = L.oct_cloud_create(C.byref(p), C.byref(h))
        check(st, None, "oct_cloud_create")
        self._h = h
        if stream is not None:
            check(L.oct_cloud_set_stream(h, C.c_void_p(stream)), h, "oct_cloud_set_stream")
        self.set_search_config(packet=packet, fp32_filter=fp32_filter, radius_lanes=radius_group,
                               knn_packet=knn_packet, knn_bucket=knn_bucket)

    # ---- checkpoints -------------------------------------------------------------
    def checkpoint(self) -> dict:
        """Everything a built cloud holds, as host arrays (np.savez-able): the sorted
        cloud (keys, perm, sorted xyz, box), the tree (export()) and its counts."""
        keys, perm, xyz = self.sorted_points()
        ck = dict(encoder=np.int32(self.encoder), max_points_leaf=np.uint32(self.max_points_leaf),
                  info=np.array([self.n, self.n_leaf, self.n_internal, self.n_total, self.max_depth_seen], np.uint64),
                  box=np.asarray(self.box, np.float64), keys=keys, perm=perm, sorted_xyz=xyz)
        ck.update(self.export())
        return ck

    @classmethod
    def from_checkpoint(cls, ck, device: int = 0, radius_group: int = 8, stream=None, packet: bool = True,
                        fp32_filter: bool = False, knn_packet: bool = True, knn_bucket: int = 256):
        """A cloud restored from checkpoint() (or its np.savez file) without sorting or building."""
        self = cls.__new__(cls)
        self._open(int(ck["encoder"]), int(ck["max_points_leaf"]), device, radius_group, stream, packet, fp32_filter,
                   knn_packet, knn_bucket)
        n, n_leaf, n_internal, n_total, depth = (int(v) for v in ck["info"])
        info = OctTreeInfo(n, n_leaf, n_internal, n_total, depth)
        arr = {k: np.ascontiguousarray(ck[k], dt) for k, dt in
               (("box", np.float64), ("keys", np.uint64), ("perm", np.uint32), ("sorted_xyz", np.float64),
                ("offsets", np.uint32), ("ranges", np.uint64), ("centers", np.float64), ("radii", np.float64),
                ("half", np.float64))}
        check(self._L.oct_tree_import(self._h, C.byref(info), *(arr[k].ctypes.data for k in
              ("box", "keys", "perm", "sorted_xyz", "offsets", "ranges", "centers", "radii", "half")), 0),
              self._h, "oct_tree_import")
        self.n, self.n_leaf, self.n_internal, self.n_total, self.max_depth_seen = n, n_leaf, n_internal, n_total, depth
        self.box = arr["box"].copy()
        return self

    @classmethod
    def from_sorted(cls, sorted_points, keys, box, encoder="hilbert", max_points_leaf: int = 128, device: int = 0,
                    **search):
        """The reference's LinearOctree(points, codes, box, enc) constructor: a cloud already in curve order with
        its ascending codes and the Box (12 doubles: center, radii, min, max) it was encoded in."""
        self = cls.__new__(cls)
        cfg = dict(radius_group=8, stream=None, packet=True, fp32_filter=False, knn_packet=True, knn_bucket=256)
        cfg.update(search)
        self._open(encoder, max_points_leaf, device, cfg["radius_group"], cfg["stream"], cfg["packet"],
                   cfg["fp32_filter"], cfg["knn_packet"], cfg["knn_bucket"])
        pts = _host_f64(sorted_points, 3)
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        b = np.ascontiguousarray(box, dtype=np.float64).reshape(12)
        self.n = int(pts.shape[0])
        assert k.shape[0] == self.n
        check(self._L.oct_set_sorted_points(self._h, pts.ctypes.data, k.ctypes.data, self.n, b.ctypes.data, 0),
              self._h, "oct_set_sorted_points")
        self.box = b.copy()
        info = OctTreeInfo()
        check(self._L.oct_build(self._h, C.byref(info)), self._h, "oct_build")
        self.n_leaf, self.n_internal, self.n_total = info.n_leaf, info.n_internal, info.n_total
        self.max_depth_seen = info.max_depth_seen
        return self

    def close(self):
        if getattr(self, "_h", None):
            self._L.oct_cloud_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_radius_group(self, lanes: int):
        check(self._L.oct_set_radius_group(self._h, int(lanes)), self._h)

    def set_search_config(self, packet: bool = True, fp32_filter: bool = False, radius_lanes: int = 8,
                          knn_packet: bool = True, knn_bucket: int = 256, two_pass: bool = False,
                          knn_estimate: int = 0, knn_group_run: int = 0):
        """Search path: packet (32 curve-ordered queries per warp) or one query per
        ``radius_lanes`` lanes; FP32 filter with FP64 re-tests (radius: leaf-relative points;
        group kNN: points relative to the box centre, FP64 only near the k-th distance; ``fp32_filter``
        True / OCT_FP32_ALL both, OCT_FP32_RADIUS or OCT_FP32_KNN one of them); kNN in groups
        of 4 queries per warp (``knn_packet``; else one warp per query); ``two_pass`` counts
        then fills instead of the one-pass packet radius search."""
        cfg = OctSearchConfig(int(bool(packet)), int(fp32_filter), int(radius_lanes), int(bool(knn_packet)),
                              int(knn_bucket))
        cfg.reserved[0] = int(bool(two_pass))
        cfg.reserved[1] = int(knn_estimate)  # kNN provisional threshold, percent; 0 default, < 0 off
        cfg.reserved[2] = int(knn_group_run)  # consecutive kNN groups per warp fetch; 0 default
        check(self._L.oct_set_search_config(self._h, C.byref(cfg)), self._h, "oct_set_search_config")

    def search_stats(self, reset: bool = False):
        """(point tests, FP64 re-tests) of the packet radius searches since the last reset."""
        a, b = C.c_uint64(), C.c_uint64()
        check(self._L.oct_search_stats(self._h, C.byref(a), C.byref(b), int(reset)), self._h)
        return a.value, b.value

    def knn_filter_stats(self, reset: bool = False):
        """(FP32 point tests, FP64 tests, band hits) of the group kNN's FP32 filter since the last reset."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(self._L.oct_knn_filter_stats(self._h, C.byref(a), C.byref(b), C.byref(c), int(reset)), self._h)
        return a.value, b.value, c.value

    # ---- sortPoints outputs ------------------------------------------------
    def sorted_points(self):
        """(keys uint64[n], perm uint32[n], sorted xyz float64[n, 3]) - the
        reordered cloud, the codes and the original ids of sortPoints."""
        n = self.n
        keys = np.zeros(n, np.uint64)
        perm = np.zeros(n, np.uint32)
        xyz = np.zeros((n, 3), np.float64)
        check(self._L.oct_encode_sort(self._h, None, keys.ctypes.data, perm.ctypes.data, xyz.ctypes.data, 0),
              self._h, "oct_encode_sort")
        return keys, perm, xyz

    def export(self):
        """The tree arrays: offsets, ranges, centers, radii (precomputedRadii), half (halfLengths)."""
        nt = self.n_total
        off = np.zeros(nt + 1, np.uint32)
        rng = np.zeros((nt, 2), np.uint64)
        ctr = np.zeros((nt, 3), np.float64)
        rad = np.zeros((22, 3), np.float64)
        half = np.zeros(3, np.float64)
        check(self._L.oct_tree_export(self._h, off.ctypes.data, rng.ctypes.data, ctr.ctypes.data, rad.ctypes.data,
                                      half.ctypes.data, 0), self._h, "oct_tree_export")
        return dict(offsets=off, ranges=rng, centers=ctr, radii=rad, half=half)

    # ---- searches -------------------------------------------------------------
    def _radii(self, centers, radius):
        if np.ndim(radius) == 0:
            return None, float(radius)
        r = np.ascontiguousarray(radius, dtype=np.float64)
        assert r.shape[0] == centers.shape[0]
        return r, 0.0

    def radius_search(self, centers, radius, kernel="square", algo="neighborsPrune"):
        """CSR result: offsets uint64[nq + 1], indices uint32 (each query ascending)."""
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        radii, r0 = self._radii(centers, radius)
        offs = np.zeros(nq + 1, np.uint64)
        total = C.c_uint64(0)
        # first call sizes the output (OCT_ERR_CAPACITY is expected when it is non-empty)
        st = L.oct_radius_search(h, KERNELS[kernel], ALGOS[algo], centers.ctypes.data, nq, _ptr(radii), r0,
                                 offs.ctypes.data, None, 0, C.byref(total), 0)
        if st == capi.OCT_ERR_CAPACITY or (st == capi.OCT_OK and total.value == 0):
            idx = np.zeros(max(1, total.value), np.uint32)
            if total.value:
                st = L.oct_radius_search(h, KERNELS[kernel], ALGOS[algo], centers.ctypes.data, nq, _ptr(radii), r0,
                                         offs.ctypes.data, idx.ctypes.data, idx.shape[0], C.byref(total), 0)
        check(st, h, "oct_radius_search")
        return offs, idx[: total.value]

    def _axes(self, centers, radii_xyz):
        r = np.ascontiguousarray(radii_xyz, dtype=np.float64)
        if r.ndim == 1:
            assert r.shape[0] == 3, "one (x, y, z) radius vector, or one per centre"
            return r, 0
        assert r.shape == (centers.shape[0], 3)
        return r, 1

    def radius_search_axes(self, centers, radii_xyz, kernel="cube", algo="neighborsPrune"):
        """The Vector-radii overloads (cube and square kernels): ``radii_xyz`` is one (x, y, z) half-extent
        vector or one per centre (nq, 3).  CSR result as radius_search."""
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        r, per = self._axes(centers, radii_xyz)
        offs = np.zeros(nq + 1, np.uint64)
        total = C.c_uint64(0)
        st = L.oct_radius_search_axes(h, KERNELS[kernel], ALGOS[algo], centers.ctypes.data, nq, r.ctypes.data, per,
                                      offs.ctypes.data, None, 0, C.byref(total), 0)
        idx = np.zeros(max(1, total.value), np.uint32)
        if st == capi.OCT_ERR_CAPACITY:
            st = L.oct_radius_search_axes(h, KERNELS[kernel], ALGOS[algo], centers.ctypes.data, nq, r.ctypes.data,
                                          per, offs.ctypes.data, idx.ctypes.data, idx.shape[0], C.byref(total), 0)
        check(st, h, "oct_radius_search_axes")
        return offs, idx[: total.value]

    def neighborsStruct_axes(self, centers, radii_xyz, kernel="cube"):
        """neighborsStruct with per-axis radii: (range offsets, pairs uint32[m, 2], numberOfPoints)."""
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        r, per = self._axes(centers, radii_xyz)
        offs = np.zeros(nq + 1, np.uint64)
        pts = np.zeros(nq, np.uint64)
        total = C.c_uint64(0)
        st = L.oct_struct_search_axes(h, KERNELS[kernel], centers.ctypes.data, nq, r.ctypes.data, per,
                                      offs.ctypes.data, None, 0, C.byref(total), pts.ctypes.data, 0)
        pairs = np.zeros((max(1, total.value), 2), np.uint32)
        if st == capi.OCT_ERR_CAPACITY:
            st = L.oct_struct_search_axes(h, KERNELS[kernel], centers.ctypes.data, nq, r.ctypes.data, per,
                                          offs.ctypes.data, pairs.ctypes.data, total.value, C.byref(total),
                                          pts.ctypes.data, 0)
        check(st, h, "oct_struct_search_axes")
        return offs, pairs[: total.value], pts

    def neighbors(self, centers, radius, kernel="square"):
        return self.radius_search(centers, radius, kernel, "neighbors")

    def neighborsPrune(self, centers, radius, kernel="square"):
        return self.radius_search(centers, radius, kernel, "neighborsPrune")

    def neighborsStruct(self, centers, radius, kernel="square"):
        """NeighborSet per query: (range offsets uint64[nq+1], pairs uint32[m, 2], numberOfPoints uint64[nq])."""
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        radii, r0 = self._radii(centers, radius)
        offs = np.zeros(nq + 1, np.uint64)
        pts = np.zeros(nq, np.uint64)
        total = C.c_uint64(0)
        st = L.oct_struct_search(h, KERNELS[kernel], centers.ctypes.data, nq, _ptr(radii), r0, offs.ctypes.data,
                                 None, 0, C.byref(total), pts.ctypes.data, 0)
        pairs = np.zeros((max(1, total.value), 2), np.uint32)
        if st == capi.OCT_ERR_CAPACITY:
            st = L.oct_struct_search(h, KERNELS[kernel], centers.ctypes.data, nq, _ptr(radii), r0, offs.ctypes.data,
                                     pairs.ctypes.data, total.value, C.byref(total), pts.ctypes.data, 0)
        check(st, h, "oct_struct_search")
        return offs, pairs[: total.value], pts

    def neighborsApprox(self, centers, radius, precision_level, upper_bound, kernel="square"):
        """neighborsApprox (linear_octree.hpp:975-1035): neighborsStruct cut below depth
        ``precision_level``; ``upper_bound`` adds the ranges of the cut octants (a superset of
        the exact set), otherwise they are dropped (a subset).  The reference's Point overloads
        take a tolerance percentage and use it as the level (converted to an unsigned integer).
        Returns (range offsets uint64[nq+1], pairs uint32[m, 2], numberOfPoints uint64[nq])."""
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        radii, r0 = self._radii(centers, radius)
        offs = np.zeros(nq + 1, np.uint64)
        pts = np.zeros(nq, np.uint64)
        total = C.c_uint64(0)
        lvl, up = int(precision_level), int(bool(upper_bound))
        st = L.oct_approx_search(h, KERNELS[kernel], centers.ctypes.data, nq, _ptr(radii), r0, lvl, up,
                                 offs.ctypes.data, None, 0, C.byref(total), pts.ctypes.data, 0)
        pairs = np.zeros((max(1, total.value), 2), np.uint32)
        if st == capi.OCT_ERR_CAPACITY:
            st = L.oct_approx_search(h, KERNELS[kernel], centers.ctypes.data, nq, _ptr(radii), r0, lvl, up,
                                     offs.ctypes.data, pairs.ctypes.data, total.value, C.byref(total),
                                     pts.ctypes.data, 0)
        check(st, h, "oct_approx_search")
        return offs, pairs[: total.value], pts

    def radius_count(self, centers, radius, kernel="square", algo="neighborsPrune"):
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        radii, r0 = self._radii(centers, radius)
        cnt = np.zeros(nq, np.uint64)
        check(L.oct_radius_count(h, KERNELS[kernel], ALGOS[algo], centers.ctypes.data, nq, _ptr(radii), r0,
                                 cnt.ctypes.data, 0), h, "oct_radius_count")
        return cnt

    def radius_hash(self, centers, radius, kernel="square", algo="neighborsPrune"):
        """(counts uint64[nq], hashes uint64[nq]): each neighbour set's size and the sum of splitmix64's
        output function over its indices (mod 2^64), without the lists.  ``centers`` may be a CUDA tensor
        (then the outputs are CUDA tensors too)."""
        L, h = self._L, self._h
        if hasattr(centers, "is_cuda") and centers.is_cuda:
            import torch

            nq = int(centers.shape[0])
            assert centers.dtype == torch.float64 and centers.is_contiguous()
            radii, r0 = (None, float(radius)) if np.isscalar(radius) else (radius, 0.0)
            cnt = torch.empty(nq, dtype=torch.int64, device=centers.device)
            hsh = torch.empty(nq, dtype=torch.int64, device=centers.device)
            _sync_current_stream()  # the cloud reads the tensors on its own stream
            check(L.oct_radius_hash(h, KERNELS[kernel], ALGOS[algo], centers.data_ptr(), nq,
                                    radii.data_ptr() if radii is not None else None, r0, cnt.data_ptr(),
                                    hsh.data_ptr(), capi.OCT_MEM_DEVICE), h, "oct_radius_hash")
            check(L.oct_synchronize(h), h, "oct_synchronize")  # the outputs are written on that stream
            return cnt, hsh
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        radii, r0 = self._radii(centers, radius)
        cnt = np.zeros(nq, np.uint64)
        hsh = np.zeros(nq, np.uint64)
        check(L.oct_radius_hash(h, KERNELS[kernel], ALGOS[algo], centers.ctypes.data, nq, _ptr(radii), r0,
                                cnt.ctypes.data, hsh.ctypes.data, 0), h, "oct_radius_hash")
        return cnt, hsh

    def knn(self, centers, k: int):
        """(idx uint32[nq, k], d2 float64[nq, k], counts uint32[nq])."""
        L, h = self._L, self._h
        centers = _host_f64(centers, 3)
        nq = centers.shape[0]
        idx = np.zeros((nq, k), np.uint32)
        d2 = np.zeros((nq, k), np.float64)
        cnt = np.zeros(nq, np.uint32)
        check(L.oct_knn(h, centers.ctypes.data, nq, k, idx.ctypes.data, d2.ctypes.data, cnt.ctypes.data, 0), h,
              "oct_knn")
        return idx, d2, cnt
