"""Bulk-load parity on the GPU: node arrays and the sorted box set of the CUDA
build, through the C ABI, are bit-identical to the oracle's and to the
reference's own GPU build (golden fixtures)."""
import glob
import os

import numpy as np
import pytest

from curtree_b200 import datasets as D
from curtree_b200.datasets import HostBoxes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    if a.shape != b.shape:
        return False
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | both_nan))


@pytest.fixture(scope="module")
def crt():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    C._lib.load()
    return C


def gpu_build(crt, b: HostBoxes, f: int):
    d = crt.BBox.from_host(b)
    rt = crt.RTree(f)
    rsz = crt.build_rtree(d, rt)
    return d, rt, rsz


def assert_tree_equal(crt, b, f, d, rt, rsz):
    sb, t = O.build(b, f)
    assert rsz == t.sz
    got = d.to_host()
    assert np.array_equal(got.id, sb.id), "sorted order differs"
    for k in ("xmin", "ymin", "xmax", "ymax"):
        assert _bits_equal(getattr(got, k), getattr(sb, k)), "permuted " + k
    if rsz:
        h = rt.to_host()
        for k in ("xmin", "ymin", "xmax", "ymax"):
            assert _bits_equal(getattr(h, k), getattr(t, k)), "node " + k
        assert np.array_equal(h.pos, t.pos)
        assert np.array_equal(h.len, t.len)


@pytest.mark.parametrize("f", [2, 3, 8, 10, 16, 32, 33, 100])
def test_build_matches_oracle_fanouts(crt, f):
    b = D.uniform_boxes(50_003, seed=30 + f)
    d, rt, rsz = gpu_build(crt, b, f)
    assert_tree_equal(crt, b, f, d, rt, rsz)
    rt.free()


@pytest.mark.parametrize("n", [1, 2, 7, 10, 11, 101, 8191, 8192, 8193, 100_000])
def test_build_small_and_tile_edges(crt, n):
    b = D.uniform_boxes(n, seed=n)
    d, rt, rsz = gpu_build(crt, b, 10)
    assert_tree_equal(crt, b, 10, d, rt, rsz)
    rt.free()


def test_build_uniform_1m(crt):
    b = D.uniform_boxes(1_000_000, seed=1)
    d, rt, rsz = gpu_build(crt, b, 10)
    assert rsz == 111_111
    assert_tree_equal(crt, b, 10, d, rt, rsz)


def test_build_clustered_with_duplicates_and_points(crt):
    b = D.clustered_boxes(3_000_000, seed=2, chunk=1_000_000)
    d, rt, rsz = gpu_build(crt, b, 10)
    assert_tree_equal(crt, b, 10, d, rt, rsz)


def test_build_raw_unit_data_is_identity(crt):
    b = D.uniform_boxes(20_000, seed=3, scale=False)
    d, rt, rsz = gpu_build(crt, b, 10)
    assert np.array_equal(d.to_host().id, np.arange(b.n))
    assert_tree_equal(crt, b, 10, d, rt, rsz)


def test_build_signed_keys_and_saturation(crt):
    rng = np.random.default_rng(12)
    n = 40_000
    cx = rng.uniform(-5000, 80000, n)
    cy = rng.uniform(-5000, 80000, n)
    w = rng.uniform(0, 30, n)
    b = HostBoxes(*(np.asarray(a, np.float32) for a in (cx - w, cy - w, cx + w, cy + w)),
                  np.arange(n, dtype=np.int32))
    d, rt, rsz = gpu_build(crt, b, 10)
    assert_tree_equal(crt, b, 10, d, rt, rsz)


def test_build_nan_and_signed_zero(crt):
    b = D.uniform_boxes(10_000, seed=13)
    b.xmin[10:20] = np.nan
    b.ymax[30:33] = np.nan
    b.xmin[40:60] = -0.0
    b.xmax[40:60] = 0.0
    d, rt, rsz = gpu_build(crt, b, 10)
    assert_tree_equal(crt, b, 10, d, rt, rsz)


def test_build_into_matches_in_place(crt):
    b = D.uniform_boxes(77_777, seed=14)
    d_in = crt.BBox.from_host(b)
    out, rt2 = crt.build_into(d_in, 16)
    # input untouched
    assert np.array_equal(d_in.to_host().id, b.id)
    d, rt, rsz = gpu_build(crt, b, 16)
    assert_tree_equal(crt, b, 16, out, rt2, rt2.sz)
    assert rt2.sz == rsz


def test_build_rejects_bad_arguments(crt):
    b = D.uniform_boxes(10, seed=1)
    d = crt.BBox.from_host(b)
    with pytest.raises(crt.CrtError):
        crt.build_rtree(d, crt.RTree(1))


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_build_matches_reference_golden(crt, path):
    z = np.load(path)
    b = HostBoxes(z["box_xmin"], z["box_ymin"], z["box_xmax"], z["box_ymax"], z["box_id"])
    f = int(z["fanout"])
    d, rt, rsz = gpu_build(crt, b, f)
    assert np.array_equal(d.to_host().id, z["sorted_id"])
    assert rsz == len(z["node_pos"])
    h = rt.to_host()
    for k in ("xmin", "ymin", "xmax", "ymax"):
        assert _bits_equal(getattr(h, k), z["node_" + k]), k
    assert np.array_equal(h.pos, z["node_pos"]) and np.array_equal(h.len, z["node_len"])
    rt.free()
