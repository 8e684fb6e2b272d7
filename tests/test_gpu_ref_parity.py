"""Full-size parity against the reference's own GPU code path, run on the same
device: its build_rtree (src/rtree_bulkload_thrust.cuh:62-179) over the
100M-box clustered set at fanout 10, and its build_rtree + bfs_frontier
(src/rtree_bfs_frontier.cuh:292-529) over 1M uniform boxes and 10k windows.
The reference runs from oracle/_ref (compiled from its sources by
`make -C oracle ref`); the tests skip where that was not built."""
import os

import numpy as np
import pytest

from curtree_b200 import datasets as D
from oracle import oracle as O
from oracle import ref_gpu as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available("ref_frontier"),
                                 reason="oracle/_ref/ref_frontier not built")]

TREE_KEYS = ("xmin", "ymin", "xmax", "ymax", "pos", "len")


@pytest.fixture(scope="module")
def crt():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    C._lib.load()
    return C


def _same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.int32), b.view(np.int32))


def test_build_100m_clustered_matches_reference_gpu(crt, tmp_path):
    """Every node MBR, pos and len, and the permuted box ids, of a 100M-box
    build equal the reference's, bit for bit (1% duplicates, 1% points)."""
    import torch
    b = D.clustered_boxes(100_000_000, seed=2)
    bfile = str(tmp_path / "boxes.crtb")
    b.write_crtb(bfile)
    t, ids, _, info = R.run("ref_frontier", "build", bfile, None, 10, str(tmp_path / "ref"))
    os.remove(bfile)
    d = crt.BBox.from_host(b)
    del b
    rt = crt.RTree(10)
    rsz = crt.build_rtree(d, rt)
    assert rsz == info["r_sz"] == len(t["pos"]) == 11_111_111
    mine = rt.to_host()
    for k in TREE_KEYS:
        assert _same_bits(t[k], getattr(mine, k)), k
    assert np.array_equal(ids, d.id.cpu().numpy())
    rt.free()
    del d
    torch.cuda.empty_cache()


def test_query_1m_10k_matches_reference_gpu(crt, tmp_path):
    """The pair set of every query form equals the reference bfs_frontier's
    on the same tree (1M uniform boxes, 10k windows, fanout 10)."""
    b = D.uniform_boxes(1_000_000, seed=1)
    q = D.uniform_windows(10_000, seed=101)
    bfile, qfile = str(tmp_path / "boxes.crtb"), str(tmp_path / "windows.crtb")
    b.write_crtb(bfile)
    q.write_crtb(qfile)
    t, ids, rp, _ = R.run("ref_frontier", "query", bfile, qfile, 10, str(tmp_path / "ref"))
    want = O.canonical_pairs(*rp)
    assert len(want[0]) > 100_000
    d = crt.BBox.from_host(b)
    rt = crt.RTree(10)
    crt.build_rtree(d, rt)
    mine = rt.to_host()
    for k in TREE_KEYS:
        assert _same_bits(t[k], getattr(mine, k)), k
    dq = crt.BBox.from_host(q)
    dp = crt.bfs_frontier(rt, d, dq)
    got = O.canonical_pairs(*dp.to_host())
    dp.free()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    for mode in (crt.CRT_QUERY_PERSISTENT, crt.CRT_QUERY_PLAIN):
        out = crt.query(rt, d, dq, mode)
        got = O.canonical_pairs(out[0].cpu().numpy(), out[1].cpu().numpy())
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), mode
    rt.free()
