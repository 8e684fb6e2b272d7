"""The C ABI surface, without a GPU: the library loads, exports every entry
point include/crtree.h declares, keeps the reference's struct layouts, and
rejects the inputs on which the reference never returns -- all on paths that
make no CUDA compute call."""
import ctypes
import os
import re

import numpy as np
import pytest

from curtree_b200 import _lib
from oracle import oracle as O

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "crtree.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(crt_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/crtree.h but not exported"
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_struct_layouts_match_reference():
    # BBOX<float>: int + 5 pointers; RTREE<float>: 2 ints + 6 pointers; IDPAIR: int + 2 pointers
    assert ctypes.sizeof(_lib.crt_bbox_f32) == 48
    assert _lib.crt_bbox_f32.xmin.offset == 8 and _lib.crt_bbox_f32.id.offset == 40
    assert ctypes.sizeof(_lib.crt_rtree_f32) == 56
    assert _lib.crt_rtree_f32.fanout.offset == 4 and _lib.crt_rtree_f32.xmin.offset == 8
    assert _lib.crt_rtree_f32.len.offset == 48
    assert ctypes.sizeof(_lib.crt_idpair) == 24 and _lib.crt_idpair.fid.offset == 8


def test_status_strings():
    L = _lib.load()
    for s in range(9):
        assert L.crt_status_string(s)
    assert L.crt_version().startswith(b"crtree")


@pytest.mark.parametrize("n,f", [(1, 10), (7, 10), (11, 10), (1_000_000, 10), (10_007, 2),
                                 (100_000_000, 16), (50_000_000, 32), (12345, 1000)])
def test_tree_size_matches_oracle_levels(n, f):
    L = _lib.load()
    lv = O.levels(n, f)
    assert L.crt_tree_size(n, f) == sum(lv)
    buf = (ctypes.c_int64 * 64)()
    assert L.crt_tree_levels(n, f, buf, 64) == len(lv)
    assert list(buf[:len(lv)]) == lv


def test_invalid_arguments_are_rejected_without_a_gpu():
    L = _lib.load()
    assert L.crt_tree_size(0, 10) == -1
    assert L.crt_tree_size(10, 1) == -1
    box = _lib.crt_bbox_f32(0, None, None, None, None, None)
    rt = _lib.crt_rtree_f32(0, 10, None, None, None, None, None, None)
    # the reference loops forever on n == 0 and on fanout == 1
    assert L.crt_build_f32(ctypes.byref(box), ctypes.byref(rt), None, None) == _lib.CRT_ERR_INVALID_ARG
    box.sz = 5
    assert L.crt_build_f32(ctypes.byref(box), ctypes.byref(rt), None, None) == _lib.CRT_ERR_INVALID_ARG
    dq = _lib.crt_idpair(0, None, None)
    assert L.crt_query_f32(None, ctypes.byref(box), ctypes.byref(box), ctypes.byref(dq), None) == \
        _lib.CRT_ERR_INVALID_ARG
    assert b"null" in L.crt_last_error() or L.crt_last_error()


def test_opts_defaults():
    o = _lib.default_opts()
    assert o.mode == _lib.CRT_QUERY_PERSISTENT and o.sort_windows == 1 and o.stage_levels == 2 and o.warps_per_window == 1


def test_device_bytes_interface():
    """Device copies in the Python layer go through torch views of raw
    device ranges (CUDA array interface), not a second CUDA runtime binding."""
    from curtree_b200.rtree import _DeviceBytes
    cai = _DeviceBytes(0x1000, 64).__cuda_array_interface__
    assert cai == {"shape": (64,), "typestr": "|u1", "data": (0x1000, False), "version": 2}
