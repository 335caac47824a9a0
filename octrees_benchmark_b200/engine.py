"""Python front end of the batched multi-cloud engine (oct_engine_* in the C ABI).

A batch is a list of requests, each a set of radius or kNN centres against one
built ``LinearOctree``.  The engine answers the whole batch in one device pass
(one sort that orders every request's centres along its cloud's curve, one
persistent launch per kernel variant, kNN on a forked stream), replayed from a
captured CUDA graph per batch shape.  Results are bitwise those of the
single-cloud calls (``LinearOctree.neighborsPrune`` / ``neighbors`` / ``knn``).

The reference has no counterpart: it answers one query per OpenMP thread
(neighbor_benchmarks.hpp:502-568).  Centres (and per-centre radii) must be CUDA
tensors on the engine's device and stay alive until the batch completes; the
engine keeps a reference to them until then.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import capi
from .capi import (ALGOS, KERNELS, OCT_MEM_DEVICE, OCT_REQ_KNN, OCT_REQ_RADIUS, OctEngineParams, OctRequest,
                   OctRequestPlace, OctSearchConfig, lib)
from .linear_octree import _sync_current_stream


@dataclass
class Request:
    """One request: ``kind`` "radius" (kernel, algo, radius or radii) or "knn" (k)."""
    cloud: object                 # LinearOctree
    kind: str                     # "radius" or "knn"
    centers: object               # CUDA tensor (nq, 3) float64
    radius: float = 0.0
    radii: object = None          # CUDA tensor (nq,) float64, or None
    kernel: str = "sphere"
    algo: str = "neighborsPrune"
    k: int = 0

    def to_c(self) -> OctRequest:
        r = OctRequest()
        r.cloud = self.cloud.handle.value if hasattr(self.cloud.handle, "value") else self.cloud.handle
        r.type = OCT_REQ_RADIUS if self.kind == "radius" else OCT_REQ_KNN
        r.kernel = KERNELS[self.kernel]
        r.algo = ALGOS[self.algo]
        r.k = int(self.k)
        nq = int(self.centers.shape[0]) if self.centers is not None else 0
        r.centers = self.centers.data_ptr() if nq else None
        r.nq = nq
        r.radii = self.radii.data_ptr() if self.radii is not None else None
        r.radius = float(self.radius)
        return r


def _engine_check(status: int, h, what: str) -> None:
    if status == capi.OCT_OK:
        return
    L = lib()
    msg = L.oct_status_string(status).decode()
    buf = C.create_string_buffer(512)
    if h:
        L.oct_engine_last_error(h, buf, 512)
        if buf.value:
            msg += ": " + buf.value.decode()
    raise capi.OctError(status, f"{what}: {msg}")


class BatchEngine:
    """Answers batches of requests over many device-resident clouds."""

    def __init__(self, device: int = 0, graph: bool = True, reserve_results: int = 0, reserve_queries: int = 0):
        L = lib()
        self._L = L
        p = OctEngineParams(device, 0 if graph else capi.OCT_ENGINE_NO_GRAPH, reserve_queries, reserve_results)
        h = C.c_void_p()
        _engine_check(L.oct_engine_create(C.byref(p), C.byref(h)), None, "oct_engine_create")
        self._h = h
        self._keep = None
        self._places = None

    def close(self):
        if getattr(self, "_h", None):
            self._L.oct_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- configuration ------------------------------------------------------
    def set_config(self, fp32_filter: bool = False, knn_bucket: int = 128, radius_blocks_per_sm: int = 0,
                   knn_blocks_per_sm: int = 0, serial: bool = False, knn_group: bool = True):
        cfg = OctSearchConfig(1, int(fp32_filter), 32, int(bool(knn_group)), int(knn_bucket))
        cfg.reserved[0] = int(radius_blocks_per_sm)
        cfg.reserved[1] = int(knn_blocks_per_sm)
        cfg.reserved[2] = int(bool(serial))
        _engine_check(self._L.oct_engine_set_config(self._h, C.byref(cfg)), self._h, "oct_engine_set_config")

    def config(self) -> dict:
        cfg = OctSearchConfig()
        _engine_check(self._L.oct_engine_get_config(self._h, C.byref(cfg)), self._h, "oct_engine_get_config")
        return dict(fp32_filter=cfg.fp32_filter, knn_bucket=cfg.knn_bucket, radius_blocks_per_sm=cfg.reserved[0],
                    knn_blocks_per_sm=cfg.reserved[1], serial=cfg.reserved[2], knn_group=cfg.knn_packet)

    def autotune(self, requests: Sequence[Request]) -> dict:
        _sync_current_stream()
        arr = (OctRequest * max(1, len(requests)))(*[r.to_c() for r in requests])
        cfg = OctSearchConfig()
        _engine_check(self._L.oct_engine_autotune(self._h, arr, len(requests), C.byref(cfg)), self._h,
                      "oct_engine_autotune")
        return self.config()

    # ---- batches --------------------------------------------------------------
    def submit(self, requests: Sequence[Request]):
        if requests:
            _sync_current_stream()  # the engine reads the centre tensors on its own stream
        arr = (OctRequest * max(1, len(requests)))(*[r.to_c() for r in requests])
        self._keep = list(requests)
        _engine_check(self._L.oct_engine_submit(self._h, arr, len(requests), None), self._h, "oct_engine_submit")
        self._n = len(requests)

    def wait(self):
        places = (OctRequestPlace * max(1, self._n))()
        total = C.c_uint64(0)
        _engine_check(self._L.oct_engine_wait(self._h, places, C.byref(total)), self._h, "oct_engine_wait")
        self._places = places
        self._keep = None
        self.radius_total = total.value
        return [places[i] for i in range(self._n)]

    def run(self, requests: Sequence[Request]):
        """Run a batch; returns the place of every request (see radius_result / knn_result)."""
        self.submit(requests)
        return self.wait()

    @property
    def last_ms(self) -> float:
        v = C.c_float(0)
        _engine_check(self._L.oct_engine_last_ms(self._h, C.byref(v)), self._h, "oct_engine_last_ms")
        return v.value

    def radius_result(self, place: OctRequestPlace):
        """(offsets uint64[nq + 1] from 0, indices uint32) of a radius request, host arrays."""
        offs = np.zeros(place.nq + 1, np.uint64)
        idx = np.zeros(max(1, place.n_results), np.uint32)
        _engine_check(self._L.oct_engine_copy_radius(self._h, C.byref(place), offs.ctypes.data, idx.ctypes.data,
                                                     idx.shape[0], 0), self._h, "oct_engine_copy_radius")
        return offs, idx[: place.n_results]

    def radius_hash_result(self, place: OctRequestPlace):
        """(counts uint64[nq], hashes uint64[nq]) of a radius request, computed on the device: each
        centre's neighbour count and the sum of splitmix64's output function over its neighbours."""
        cnt = np.zeros(place.nq, np.uint64)
        hsh = np.zeros(place.nq, np.uint64)
        _engine_check(self._L.oct_engine_copy_radius_hash(self._h, C.byref(place), cnt.ctypes.data,
                                                          hsh.ctypes.data, 0), self._h, "oct_engine_copy_radius_hash")
        return cnt, hsh

    def knn_result(self, place: OctRequestPlace, k: int):
        """(idx uint32[nq, k], d2 float64[nq, k], counts uint32[nq]) of a kNN request, host arrays."""
        idx = np.zeros((place.nq, k), np.uint32)
        d2 = np.zeros((place.nq, k), np.float64)
        cnt = np.zeros(place.nq, np.uint32)
        _engine_check(self._L.oct_engine_copy_knn(self._h, C.byref(place), k, idx.ctypes.data, d2.ctypes.data,
                                                  cnt.ctypes.data, 0), self._h, "oct_engine_copy_knn")
        return idx, d2, cnt

    def outputs(self):
        """Device pointers (offsets, indices, knn_idx, knn_d2, knn_counts) of the last batch."""
        ptrs = [C.c_void_p() for _ in range(5)]
        _engine_check(self._L.oct_engine_outputs(self._h, *[C.byref(p) for p in ptrs]), self._h,
                      "oct_engine_outputs")
        return tuple(p.value for p in ptrs)
