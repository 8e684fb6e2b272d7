"""ctypes binding of the crtree C ABI (include/crtree.h).

The shared library is built in-tree (curtree_b200/libcrtree.so, by
`make -C curtree_b200/csrc` or `__graft_entry__.build()`).  Importing the
bindings without it raises: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcrtree.so")

CRT_OK = 0
CRT_ERR_INVALID_ARG = 1
CRT_ERR_OOM = 2
CRT_ERR_OVERFLOW_INT32 = 3
CRT_ERR_OUTPUT_OVERFLOW = 4
CRT_ERR_DEVICE_TIMEOUT = 5
CRT_ERR_CUDA = 6
CRT_ERR_NOT_SUPPORTED = 7
CRT_ERR_BUSY = 8

CRT_QUERY_PERSISTENT = 0
CRT_QUERY_PLAIN = 1

_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


class crt_bbox_f32(ctypes.Structure):
    """BBOX<float> (src/rtree.h:3-11)."""
    _fields_ = [("sz", ctypes.c_int), ("xmin", ctypes.c_void_p), ("ymin", ctypes.c_void_p),
                ("xmax", ctypes.c_void_p), ("ymax", ctypes.c_void_p), ("id", ctypes.c_void_p)]


class crt_rtree_f32(ctypes.Structure):
    """RTREE<float> (src/rtree.h:13-23)."""
    _fields_ = [("sz", ctypes.c_int), ("fanout", ctypes.c_int), ("xmin", ctypes.c_void_p),
                ("ymin", ctypes.c_void_p), ("xmax", ctypes.c_void_p), ("ymax", ctypes.c_void_p),
                ("pos", ctypes.c_void_p), ("len", ctypes.c_void_p)]


class crt_idpair(ctypes.Structure):
    """IDPAIR (src/rtree.h:25-29)."""
    _fields_ = [("sz", ctypes.c_int), ("fid", ctypes.c_void_p), ("tid", ctypes.c_void_p)]


class crt_query_opts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("sort_windows", ctypes.c_int),
                ("stage_levels", ctypes.c_int), ("warps_per_cta", ctypes.c_int),
                ("chunk", ctypes.c_int), ("no_contain", ctypes.c_int),
                ("warps_per_window", ctypes.c_int), ("reserved", ctypes.c_int * 1)]


class crt_query_result(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int64), ("required", ctypes.c_int64),
                ("overflow", ctypes.c_int32), ("error", ctypes.c_int32),
                ("reserved", ctypes.c_int64 * 5)]


class crt_server_opts(ctypes.Structure):
    _fields_ = [("arena_bytes", ctypes.c_int64), ("max_requests", ctypes.c_int),
                ("max_trees", ctypes.c_int), ("pairs_per_window", ctypes.c_double),
                ("output_slack", ctypes.c_double), ("idle_ms", ctypes.c_int),
                ("device_wait_us", ctypes.c_int64), ("reserved", ctypes.c_int * 4)]


class crt_server_completion(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_int64), ("tree_id", ctypes.c_int), ("status", ctypes.c_int),
                ("nq", ctypes.c_int64), ("count", ctypes.c_int64), ("d_fid", ctypes.c_void_p),
                ("d_tid", ctypes.c_void_p), ("submit_time_s", ctypes.c_double),
                ("complete_time_s", ctypes.c_double), ("retries", ctypes.c_int),
                ("reserved", ctypes.c_int)]


assert ctypes.sizeof(crt_bbox_f32) == 48
assert ctypes.sizeof(crt_rtree_f32) == 56
assert ctypes.sizeof(crt_idpair) == 24
assert ctypes.sizeof(crt_query_result) == 64

# Every symbol include/crtree.h declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
SIGNATURES = {
    "crt_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "crt_last_error": (ctypes.c_char_p, []),
    "crt_version": (ctypes.c_char_p, []),
    "crt_kernel_launches": (ctypes.c_uint64, []),
    "crt_build_f32": (ctypes.c_int, [ctypes.POINTER(crt_bbox_f32), ctypes.POINTER(crt_rtree_f32),
                                     _vp, ctypes.POINTER(_i32)]),
    "crt_query_f32": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32), ctypes.POINTER(crt_bbox_f32),
                                     ctypes.POINTER(crt_bbox_f32), ctypes.POINTER(crt_idpair),
                                     _vp]),
    "crt_query_thrust_f32": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32),
                                            ctypes.POINTER(crt_bbox_f32),
                                            ctypes.POINTER(crt_bbox_f32),
                                            ctypes.POINTER(crt_idpair), _vp]),
    "crt_rtree_free": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32)]),
    "crt_idpair_free": (ctypes.c_int, [ctypes.POINTER(crt_idpair)]),
    "crt_build_into_f32": (ctypes.c_int, [ctypes.POINTER(crt_bbox_f32),
                                          ctypes.POINTER(crt_bbox_f32),
                                          ctypes.POINTER(crt_rtree_f32), _vp]),
    "crt_tree_size": (_i64, [_i64, ctypes.c_int]),
    "crt_tree_levels": (ctypes.c_int, [_i64, ctypes.c_int, ctypes.POINTER(_i64), ctypes.c_int]),
    "crt_query_opts_default": (None, [ctypes.POINTER(crt_query_opts)]),
    "crt_query_into_f32": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32),
                                          ctypes.POINTER(crt_bbox_f32),
                                          ctypes.POINTER(crt_bbox_f32), _vp, _vp, _i64, _vp, _vp,
                                          ctypes.POINTER(crt_query_opts), _vp]),
    "crt_query_capacity": (_i64, [_i64, ctypes.POINTER(crt_query_opts)]),
    "crt_pairs_canonicalize": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "crt_pairs_digest": (ctypes.c_int, [_vp, _vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp]),
    "crt_read_mbr_csv": (ctypes.c_int, [ctypes.c_char_p, _i64, ctypes.c_float, _vp, _vp, _vp, _vp,
                                        _vp, ctypes.POINTER(_i64)]),
    "crt_read_mbr_csv_device": (ctypes.c_int, [ctypes.c_char_p, _i64, ctypes.c_float,
                                               ctypes.POINTER(crt_bbox_f32), ctypes.POINTER(_i64),
                                               _vp]),
    "crt_read_mbr_bin_device": (ctypes.c_int, [ctypes.c_char_p, _i64, ctypes.c_float,
                                               ctypes.POINTER(crt_bbox_f32), ctypes.POINTER(_i64),
                                               _vp]),
    "crt_parse_mbr_csv_device": (ctypes.c_int, [_vp, _i64, _i64, ctypes.c_float, _vp, _vp, _vp,
                                                _vp, _vp, ctypes.POINTER(_i64), _vp]),
    "crt_tree_save": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(crt_rtree_f32),
                                     ctypes.POINTER(crt_bbox_f32)]),
    "crt_tree_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(crt_rtree_f32),
                                     ctypes.POINTER(crt_bbox_f32)]),
    "crt_bbox_free": (ctypes.c_int, [ctypes.POINTER(crt_bbox_f32)]),
    "crt_query_sync_f32": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32),
                                          ctypes.POINTER(crt_bbox_f32),
                                          ctypes.POINTER(crt_bbox_f32), _vp, _vp, _i64,
                                          ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                          ctypes.POINTER(crt_query_opts), _vp]),
    "crt_plan_create": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32), ctypes.POINTER(crt_bbox_f32),
                                       ctypes.POINTER(crt_bbox_f32), _i64, _vp, _vp, _i64, _vp,
                                       ctypes.POINTER(crt_query_opts), _vp,
                                       ctypes.POINTER(_vp)]),
    "crt_query_plain_noalloc_f32": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32),
                                                   ctypes.POINTER(crt_bbox_f32),
                                                   ctypes.POINTER(crt_bbox_f32), _vp, _vp, _i64,
                                                   _vp, _vp]),
    "crt_query_stats_f32": (ctypes.c_int, [ctypes.POINTER(crt_rtree_f32),
                                           ctypes.POINTER(crt_bbox_f32),
                                           ctypes.POINTER(crt_bbox_f32), _vp, _vp,
                                           ctypes.POINTER(_i64), _vp]),
    "crt_plan_set_nq": (ctypes.c_int, [_vp, _i64, _vp]),
    "crt_plan_launch": (ctypes.c_int, [_vp, _vp]),
    "crt_plan_destroy": (ctypes.c_int, [_vp]),
    "crt_server_opts_default": (None, [ctypes.POINTER(crt_server_opts)]),
    "crt_server_create": (ctypes.c_int, [ctypes.POINTER(crt_server_opts), ctypes.POINTER(_vp)]),
    "crt_server_add_tree": (ctypes.c_int, [_vp, ctypes.POINTER(crt_rtree_f32),
                                           ctypes.POINTER(crt_bbox_f32), ctypes.POINTER(ctypes.c_int)]),
    "crt_server_submit": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _i64,
                                         ctypes.POINTER(_i64)]),
    "crt_server_poll": (ctypes.c_int, [_vp, ctypes.POINTER(crt_server_completion), ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "crt_server_release": (ctypes.c_int, [_vp, _i64]),
    "crt_server_stats": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                        ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "crt_server_destroy": (ctypes.c_int, [_vp]),
    "crt_profile_enable": (None, [ctypes.c_int]),
    "crt_profile_collect": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(_i64)]),
}

_lib = None


class CrtError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        lib = _lib
        detail = lib.crt_last_error().decode() if lib is not None else ""
        name = lib.crt_status_string(status).decode() if lib is not None else str(status)
        super().__init__(f"{where}: {name} ({status}): {detail}")


def load():
    """Load libcrtree.so and bind every exported entry point."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C curtree_b200/csrc` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != CRT_OK:
        raise CrtError(status, where)


def default_opts(**kw) -> crt_query_opts:
    o = crt_query_opts()
    load().crt_query_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
