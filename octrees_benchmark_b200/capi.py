"""ctypes binding of the C ABI in include/octree_b200.h (liboctree_b200.so).

Loading fails loudly when the library has not been built: there is no CPU
fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liboctree_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "octree_b200.h")

OCT_OK = 0
OCT_ERR_INVALID_ARG = 1
OCT_ERR_CUDA = 2
OCT_ERR_OUT_OF_MEMORY = 3
OCT_ERR_STATE = 4
OCT_ERR_CAPACITY = 5
OCT_ERR_DEVICE_LIMIT = 6
OCT_ERR_NO_DEVICE = 7
OCT_MEM_DEVICE = 0x1
OCT_CLOUD_SORT_8PASS = 0x1
OCT_NOALLOC_MAX_POINTS = 1 << 18

ENCODERS = {"morton": 1, "mort": 1, "hilbert": 5, "hilb": 5, 1: 1, 5: 5}
KERNELS = {"circle": 0, "sphere": 1, "square": 2, "cube": 3, 0: 0, 1: 1, 2: 2, 3: 3}
ALGOS = {"neighbors": 1, "neighborsPrune": 2, "prune": 2, "neighborsStruct": 3, "struct": 3, 1: 1, 2: 2, 3: 3}
OCT_NEIGHBORS_APPROX = 4  # oct_approx_search (SearchAlgo::NEIGHBORS_APPROX)


class OctParams(C.Structure):
    _fields_ = [("max_points_leaf", C.c_uint32), ("encoder", C.c_int32), ("device", C.c_int32),
                ("flags", C.c_uint32)]


class OctSearchConfig(C.Structure):
    _fields_ = [("packet", C.c_int32), ("fp32_filter", C.c_int32), ("radius_lanes", C.c_int32),
                ("knn_packet", C.c_int32), ("knn_bucket", C.c_int32), ("reserved", C.c_int32 * 3)]


class OctTreeInfo(C.Structure):
    _fields_ = [("n_points", C.c_uint64), ("n_leaf", C.c_uint32), ("n_internal", C.c_uint32),
                ("n_total", C.c_uint32), ("max_depth_seen", C.c_uint32)]


OCT_ENGINE_NO_GRAPH = 0x1
OCT_REQ_RADIUS = 0
OCT_REQ_KNN = 1


class OctEngineParams(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32), ("reserve_queries", C.c_uint64),
                ("reserve_results", C.c_uint64)]


class OctRequest(C.Structure):
    _fields_ = [("cloud", C.c_void_p), ("type", C.c_int32), ("kernel", C.c_int32), ("algo", C.c_int32),
                ("k", C.c_uint32), ("centers", C.c_void_p), ("nq", C.c_uint64), ("radii", C.c_void_p),
                ("radius", C.c_double)]


class OctRequestPlace(C.Structure):
    _fields_ = [("q_begin", C.c_uint64), ("out_begin", C.c_uint64), ("nq", C.c_uint64),
                ("n_results", C.c_uint64)]


OCT_SERVER_PLAIN = 0x1
OCT_SERVER_FIFO = 0x2
OCT_SERVER_NO_GRAPH = 0x4
OCT_FP32_ALL = 1
OCT_FP32_RADIUS = 2
OCT_FP32_KNN = 3
OCT_CLOUD_OWNED = 0x1


class OctServerParams(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32), ("slots", C.c_uint32),
                ("max_batch_requests", C.c_uint32), ("max_batch_queries", C.c_uint64), ("hbm_budget", C.c_uint64),
                ("max_wait_ms", C.c_double)]


class OctCompletion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("type", C.c_int32), ("nq", C.c_uint64),
                ("n_results", C.c_uint64), ("queue_ms", C.c_double), ("latency_ms", C.c_double)]


class OctServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("admission_stalls", C.c_uint64), ("evictions", C.c_uint64), ("queries", C.c_uint64),
                ("cloud_bytes", C.c_uint64), ("inflight_bytes", C.c_uint64), ("peak_bytes", C.c_uint64),
                ("queued", C.c_uint32), ("in_flight", C.c_uint32), ("max_submit_ms", C.c_double),
                ("max_finish_ms", C.c_double)]


class OctError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


_lib = None

_vp = C.c_void_p
_u64 = C.c_uint64
_u32 = C.c_uint32
_int = C.c_int
_dbl = C.c_double

SIGNATURES = {
    "oct_abi_version": ([], _int),
    "oct_status_string": ([_int], C.c_char_p),
    "oct_cloud_create": ([C.POINTER(OctParams), C.POINTER(_vp)], _int),
    "oct_cloud_destroy": ([_vp], _int),
    "oct_cloud_set_stream": ([_vp, _vp], _int),
    "oct_last_error": ([_vp, C.c_char_p, C.c_size_t], _int),
    "oct_synchronize": ([_vp], _int),
    "oct_set_radius_group": ([_vp, _int], _int),
    "oct_set_search_config": ([_vp, C.POINTER(OctSearchConfig)], _int),
    "oct_search_stats": ([_vp, C.POINTER(_u64), C.POINTER(_u64), _int], _int),
    "oct_knn_filter_stats": ([_vp, C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64), _int], _int),
    "oct_set_points": ([_vp, _vp, _u64, _u32], _int),
    "oct_encode_sort": ([_vp, _vp, _vp, _vp, _vp, _u32], _int),
    "oct_build": ([_vp, C.POINTER(OctTreeInfo)], _int),
    "oct_tree_export": ([_vp, _vp, _vp, _vp, _vp, _vp, _u32], _int),
    "oct_radius_search": ([_vp, _int, _int, _vp, _u64, _vp, _dbl, _vp, _vp, _u64, C.POINTER(_u64), _u32], _int),
    "oct_radius_count": ([_vp, _int, _int, _vp, _u64, _vp, _dbl, _vp, _u32], _int),
    "oct_struct_search": ([_vp, _int, _vp, _u64, _vp, _dbl, _vp, _vp, _u64, C.POINTER(_u64), _vp, _u32], _int),
    "oct_search_timing": ([_vp, _int], _int),
    "oct_search_kernel_times": ([_vp, C.POINTER(_dbl), C.POINTER(_u64), C.POINTER(_dbl), C.POINTER(_u64), _int],
                                _int),
    "oct_set_sorted_points": ([_vp, _vp, _vp, _u64, _vp, _u32], _int),
    "oct_radius_search_axes": ([_vp, _int, _int, _vp, _u64, _vp, _int, _vp, _vp, _u64, C.POINTER(_u64), _u32], _int),
    "oct_struct_search_axes": ([_vp, _int, _vp, _u64, _vp, _int, _vp, _vp, _u64, C.POINTER(_u64), _vp, _u32], _int),
    "oct_approx_search": ([_vp, _int, _vp, _u64, _vp, _dbl, _u32, _int, _vp, _vp, _u64, C.POINTER(_u64), _vp, _u32],
                          _int),
    "oct_tree_import": ([_vp, C.POINTER(OctTreeInfo), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32], _int),
    "oct_knn": ([_vp, _vp, _u64, _u32, _vp, _vp, _vp, _u32], _int),
    "oct_encode_sort_noalloc": ([_int, _vp, _u64, _vp, _vp, _vp, _vp], _int),
    "oct_engine_create": ([C.POINTER(OctEngineParams), C.POINTER(_vp)], _int),
    "oct_engine_destroy": ([_vp], _int),
    "oct_engine_set_stream": ([_vp, _vp], _int),
    "oct_engine_last_error": ([_vp, C.c_char_p, C.c_size_t], _int),
    "oct_engine_set_config": ([_vp, C.POINTER(OctSearchConfig)], _int),
    "oct_engine_get_config": ([_vp, C.POINTER(OctSearchConfig)], _int),
    "oct_engine_submit": ([_vp, C.POINTER(OctRequest), _u32, C.POINTER(OctRequestPlace)], _int),
    "oct_engine_wait": ([_vp, C.POINTER(OctRequestPlace), C.POINTER(_u64)], _int),
    "oct_engine_run": ([_vp, C.POINTER(OctRequest), _u32, C.POINTER(OctRequestPlace), C.POINTER(_u64)], _int),
    "oct_engine_outputs": ([_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)],
                           _int),
    "oct_engine_copy_radius": ([_vp, C.POINTER(OctRequestPlace), _vp, _vp, _u64, _u32], _int),
    "oct_engine_copy_knn": ([_vp, C.POINTER(OctRequestPlace), _u32, _vp, _vp, _vp, _u32], _int),
    "oct_engine_autotune": ([_vp, C.POINTER(OctRequest), _u32, C.POINTER(OctSearchConfig)], _int),
    "oct_engine_last_ms": ([_vp, C.POINTER(C.c_float)], _int),
    "oct_engine_ready": ([_vp, C.POINTER(_int)], _int),
    "oct_engine_memory": ([_vp, C.POINTER(_u64)], _int),
    "oct_cloud_memory": ([_vp, C.POINTER(_u64)], _int),
    "oct_trim_cloud_memory": ([_int], _int),
    "oct_radius_hash": ([_vp, _int, _int, _vp, _u64, _vp, _dbl, _vp, _vp, _u32], _int),
    "oct_engine_copy_radius_hash": ([_vp, _vp, _vp, _vp, _u32], _int),
    "oct_device_wait_probe": ([_int, C.c_uint32, C.POINTER(C.c_uint32)], _int),
    "oct_server_create": ([C.POINTER(OctServerParams), C.POINTER(_vp)], _int),
    "oct_server_destroy": ([_vp], _int),
    "oct_server_last_error": ([_vp, C.c_char_p, C.c_size_t], _int),
    "oct_server_set_config": ([_vp, C.POINTER(OctSearchConfig)], _int),
    "oct_server_add_cloud": ([_vp, _vp, _u32], _int),
    "oct_server_remove_cloud": ([_vp, _vp], _int),
    "oct_server_submit": ([_vp, C.POINTER(OctRequest), C.POINTER(_u64)], _int),
    "oct_server_poll": ([_vp, C.POINTER(OctCompletion), _u32, C.POINTER(_u32), C.c_int32], _int),
    "oct_server_copy_radius": ([_vp, _u64, _vp, _vp, _u64, _u32], _int),
    "oct_server_copy_knn": ([_vp, _u64, _vp, _vp, _vp, _u32], _int),
    "oct_server_release": ([_vp, _u64], _int),
    "oct_server_get_stats": ([_vp, C.POINTER(OctServerStats)], _int),
}


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions declared in include/octree_b200.h."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(oct_[a-z_0-9]+)\s*\(", txt)))


def lib() -> C.CDLL:
    """The loaded device library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m octrees_benchmark_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int, cloud=None, what: str = "") -> None:
    if status == OCT_OK:
        return
    L = lib()
    msg = L.oct_status_string(status).decode()
    if cloud:
        buf = C.create_string_buffer(512)
        L.oct_last_error(cloud, buf, 512)
        if buf.value:
            msg += ": " + buf.value.decode()
    raise OctError(status, f"{what}: {msg}" if what else msg)
