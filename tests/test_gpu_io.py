"""GPU canonicalisation of pair lists and tree persistence, through the C ABI."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from curtree_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def crt():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    C._lib.load()
    return C


@pytest.mark.parametrize("n", [0, 1, 2, 1000, 8191, 8193, 2_000_003])
def test_canonicalize_random_pairs(crt, n):
    import torch
    rng = np.random.default_rng(n)
    fid = rng.integers(-2**31, 2**31 - 1, n).astype(np.int32)
    tid = rng.integers(-1000, 1000, n).astype(np.int32)
    fid[: n // 3] = fid[0] if n else 0  # many equal box ids
    f = torch.from_numpy(fid).cuda()
    t = torch.from_numpy(tid).cuda()
    crt.canonicalize(f, t)
    o = np.lexsort((fid, tid))
    assert np.array_equal(f.cpu().numpy(), fid[o]) and np.array_equal(t.cpu().numpy(), tid[o])


def test_canonicalized_query_output_is_the_reference_order(crt):
    b = D.uniform_boxes(500_000, seed=95)
    q = D.mixed_windows(5000, b, seed=195, lo=1e-5, hi=2e-2)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(10)
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    fid, tid = crt.query(rt, d, dq)
    crt.canonicalize(fid, tid)
    sb, t = O.build(b, 10)
    want = O.canonical_pairs(*O.tree_query_pairs(t, sb, q))
    assert np.array_equal(fid.cpu().numpy(), want[0]) and np.array_equal(tid.cpu().numpy(), want[1])


def test_tree_save_load_round_trip(crt):
    from curtree_b200 import _lib
    L = _lib.load()
    b = D.clustered_boxes(300_000, seed=96, chunk=100_000)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(16)
    crt.build_rtree(d, rt)
    q = D.mixed_windows(3000, b, seed=196)
    dq = crt.BBox.from_host(q)
    want = O.canonical_pairs(*[x.cpu().numpy() for x in crt.query(rt, d, dq)])
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "tree.crt").encode()
        rb = d.c()
        assert L.crt_tree_save(path, ctypes.byref(rt.s), ctypes.byref(rb)) == 0
        rt2 = crt.RTree(0)
        bx = _lib.crt_bbox_f32()
        assert L.crt_tree_load(path, ctypes.byref(rt2.s), ctypes.byref(bx)) == 0, L.crt_last_error()
        rt2.owned = True
        assert rt2.sz == rt.sz and rt2.fanout == 16 and bx.sz == b.n
        h1, h2 = rt.to_host(), rt2.to_host()
        for k in ("xmin", "ymin", "xmax", "ymax", "pos", "len"):
            assert np.array_equal(getattr(h1, k).view(np.uint32), getattr(h2, k).view(np.uint32))
        # query the loaded tree through raw pointers
        from curtree_b200.rtree import IDPair
        out = IDPair()
        qb = dq.c()
        assert L.crt_query_f32(ctypes.byref(rt2.s), ctypes.byref(bx), ctypes.byref(qb),
                               ctypes.byref(out.s), None) == 0
        got = O.canonical_pairs(*out.to_host())
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        out.free()
        assert L.crt_bbox_free(ctypes.byref(bx)) == 0
        rt2.free()
        # damaged files are rejected
        with open(path, "r+b") as f:
            f.seek(0)
            f.write(b"XXXX")
        assert L.crt_tree_load(path, ctypes.byref(rt2.s), ctypes.byref(bx)) == _lib.CRT_ERR_INVALID_ARG
