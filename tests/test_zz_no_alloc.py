"""The allocation-free plain query (crt_query_plain_noalloc_f32), through the
C ABI, against the plain query that allocates its scratch
(crt_query_into_f32, CRT_QUERY_PLAIN).

It exists for callers that cannot allocate device memory while they run --
a process whose device memory belongs to another allocator or budget, or a
loop that cannot take cudaMalloc's implicit synchronisation -- so its scratch
is a fixed device array inside the library.  Both entry points produce the
same pairs in the same order (grouped by window), so the outputs must be
identical, element for element, on two calls in a row (the second call
reuses the array the first one left behind).  This file is collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from curtree_b200 import datasets as D

pytestmark = pytest.mark.gpu


def test_noalloc_plain_query_matches_allocating_plain_query():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    from curtree_b200 import _lib
    from curtree_b200.rtree import _stream_handle

    L = _lib.load()
    b = D.uniform_boxes(300_000, seed=90)
    d = C.BBox.from_host(b)
    rt = C.RTree(10)
    C.build_rtree(d, rt)
    q = D.mixed_windows(20_000, b, seed=190, lo=1e-5, hi=5e-2)
    dq = C.BBox.from_host(q)

    # reference output: the allocating plain query
    want_fid, want_tid, _ = C.query(rt, d, dq, mode=C.CRT_QUERY_PLAIN)
    n = want_fid.numel()
    assert n > 100_000
    want_fid = want_fid.cpu().numpy()
    want_tid = want_tid.cpu().numpy()

    rb, qb = d.c(), dq.c()
    for call in range(2):
        fid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        tid = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        res = C.new_result_block()
        st = L.crt_query_plain_noalloc_f32(ctypes.byref(rt.s), ctypes.byref(rb), ctypes.byref(qb),
                                           fid.data_ptr(), tid.data_ptr(), n, res.data_ptr(),
                                           _stream_handle(None))
        assert st == _lib.CRT_OK, L.crt_last_error()
        r = C.read_result(res)
        assert r["error"] == 0 and r["overflow"] == 0 and r["count"] == n, (call, r)
        assert np.array_equal(fid.cpu().numpy(), want_fid), call
        assert np.array_equal(tid.cpu().numpy(), want_tid), call

    # more windows than the fixed scratch holds: a clear error, nothing launched
    big = D.uniform_windows(70_000, seed=191)
    dbig = C.BBox.from_host(big)
    bb = dbig.c()
    res = C.new_result_block()
    st = L.crt_query_plain_noalloc_f32(ctypes.byref(rt.s), ctypes.byref(rb), ctypes.byref(bb),
                                       None, None, 0, res.data_ptr(), _stream_handle(None))
    assert st == _lib.CRT_ERR_INVALID_ARG
    assert b"65536" in L.crt_last_error()


def test_noalloc_plain_query_matches_oracle_and_reports_overflow():
    """The allocation-free plain query against the oracle's pairs (bit-exact
    canonical sets) at the 65536-window limit, and with an output one pair too
    small: the result block reports overflow and the exact pair count, and a
    retry at that size succeeds -- on the same shared scratch."""
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    from curtree_b200 import _lib
    from curtree_b200.rtree import _stream_handle
    from oracle import oracle as O

    L = _lib.load()
    b = D.clustered_boxes(200_000, seed=92)
    d = C.BBox.from_host(b)
    rt = C.RTree(16)
    C.build_rtree(d, rt)
    q = D.mixed_windows(65_536, b, seed=192, lo=1e-5, hi=2e-2)
    dq = C.BBox.from_host(q)
    sb, t = O.build(b, 16)
    want = O.canonical_pairs(*O.tree_query_pairs(t, sb, q))
    n = len(want[0])
    assert n > 50_000

    rb, qb = d.c(), dq.c()

    def call(cap):
        fid = torch.full((max(cap, 1),), -1, dtype=torch.int32, device="cuda")
        tid = torch.full((max(cap, 1),), -1, dtype=torch.int32, device="cuda")
        res = C.new_result_block()
        st = L.crt_query_plain_noalloc_f32(ctypes.byref(rt.s), ctypes.byref(rb), ctypes.byref(qb),
                                           fid.data_ptr(), tid.data_ptr(), cap, res.data_ptr(),
                                           _stream_handle(None))
        assert st == _lib.CRT_OK, L.crt_last_error()
        return fid, tid, C.read_result(res)

    fid, tid, r = call(n - 1)
    assert r["overflow"] == 1 and r["required"] == n and r["count"] == 0 and r["error"] == 0, r
    fid, tid, r = call(n)
    assert r["overflow"] == 0 and r["count"] == n and r["error"] == 0, r
    got = O.canonical_pairs(fid.cpu().numpy(), tid.cpu().numpy())
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    # grouped by window, in window order
    assert np.all(np.diff(tid.cpu().numpy()) >= 0)
