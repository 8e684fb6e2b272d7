"""Window-query parity on the GPU: every form (drop-in bfs_frontier /
bfs_thrust, plain, persistent, graph plan) returns exactly the oracle's hit
pairs, through the C ABI, on the reference's edge cases."""
import glob
import os

import numpy as np
import pytest

from curtree_b200 import datasets as D
from curtree_b200.datasets import HostBoxes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def crt():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    C._lib.load()
    return C


def canon(fid, tid):
    fid = fid.cpu().numpy() if hasattr(fid, "cpu") else np.asarray(fid)
    tid = tid.cpu().numpy() if hasattr(tid, "cpu") else np.asarray(tid)
    return O.canonical_pairs(fid, tid)


def setup(crt, b, q, f=10):
    d = crt.BBox.from_host(b)
    rt = crt.RTree(f)
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    sb, t = O.build(b, f)
    want = O.canonical_pairs(*O.tree_query_pairs(t, sb, q))
    return d, rt, dq, want


def all_forms(crt, d, rt, dq):
    out = {}
    p = crt.bfs_frontier(rt, d, dq)
    out["frontier"] = canon(*p.to_host())
    p.free()
    p = crt.bfs_thrust(rt, d, dq)
    out["thrust"] = canon(*p.to_host())
    p.free()
    out["plain"] = canon(*crt.query(rt, d, dq, mode=crt.CRT_QUERY_PLAIN)[:2])
    out["persistent"] = canon(*crt.query(rt, d, dq))
    out["persistent_unsorted"] = canon(*crt.query(rt, d, dq, sort_windows=0))
    out["persistent_unstaged"] = canon(*crt.query(rt, d, dq, stage_levels=0))
    out["persistent_small_chunk"] = canon(*crt.query(rt, d, dq, chunk=64))
    out["persistent_2_warps_per_window"] = canon(*crt.query(rt, d, dq, warps_per_window=2))
    out["persistent_4_warps_per_window"] = canon(*crt.query(rt, d, dq, warps_per_window=4,
                                                           warps_per_cta=32))
    out["persistent_staged_4_levels"] = canon(*crt.query(rt, d, dq, stage_levels=4))
    return out


def assert_all(out, want):
    for k, v in out.items():
        assert np.array_equal(v[0], want[0]) and np.array_equal(v[1], want[1]), k


@pytest.mark.parametrize("f", [2, 3, 8, 10, 16, 32, 40])
def test_query_fanouts(crt, f):
    b = D.uniform_boxes(60_000, seed=40 + f)
    q = D.mixed_windows(2000, b, seed=140 + f, lo=1e-4, hi=5e-2)
    d, rt, dq, want = setup(crt, b, q, f)
    assert len(want[0]) > 0
    assert_all(all_forms(crt, d, rt, dq), want)


def test_query_uniform_1m_10k_matches_brute_force(crt):
    """1M boxes, 10k windows, fanout 10: pairs equal the brute force's."""
    b = D.uniform_boxes(1_000_000, seed=1)
    q = D.uniform_windows(10_000, seed=101)
    d, rt, dq, want = setup(crt, b, q, 10)
    got = canon(*crt.query(rt, d, dq))
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    c, h = O.nested_loop_stats(q, b)
    gc, gh = O.pair_hashes(got[0], got[1], q.n)
    assert np.array_equal(gc, c) and np.array_equal(gh, h)
    p = crt.bfs_frontier(rt, d, dq)
    g2 = canon(*p.to_host())
    assert np.array_equal(g2[0], want[0]) and np.array_equal(g2[1], want[1])


def test_query_touching_edges_points_and_duplicates(crt):
    b = D.uniform_boxes(20_000, seed=50)
    b.xmax[::9] = b.xmin[::9]  # zero-width
    b.ymax[::9] = b.ymin[::9]
    for a in (b.xmin, b.ymin, b.xmax, b.ymax):
        a[500:700] = a[499]  # duplicates
    q = b.take(np.arange(0, 20_000, 37))  # windows equal to boxes: touching edges
    q.id = np.arange(q.n, dtype=np.int32)
    pts = D.uniform_windows(300, seed=150, max_side=0.0)  # point windows
    q = HostBoxes.concat([q, pts])
    q.id = np.arange(q.n, dtype=np.int32)
    d, rt, dq, want = setup(crt, b, q, 10)
    assert_all(all_forms(crt, d, rt, dq), want)


def test_query_all_miss_and_empty_batches(crt):
    b = D.uniform_boxes(10_000, seed=51)
    far = HostBoxes(*(np.full(100, v, np.float32) for v in (1e6, 1e6, 1e6 + 1, 1e6 + 1)),
                    np.arange(100, dtype=np.int32))
    d, rt, dq, want = setup(crt, b, far, 10)
    assert len(want[0]) == 0
    assert_all(all_forms(crt, d, rt, dq), want)
    empty = HostBoxes(*(np.zeros(0, np.float32) for _ in range(4)), np.zeros(0, np.int32))
    de = crt.BBox.from_host(empty)
    fid, tid = crt.query(rt, d, de)
    assert fid.numel() == 0
    fid, tid, offs = crt.query(rt, d, de, mode=crt.CRT_QUERY_PLAIN)
    assert fid.numel() == 0


def test_query_one_box_tree(crt):
    b = D.uniform_boxes(1, seed=52)
    q = HostBoxes.concat([b, D.uniform_windows(50, seed=152, max_side=0.5)])
    q.id = np.arange(q.n, dtype=np.int32)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(10)
    assert crt.build_rtree(d, rt) == 0
    dq = crt.BBox.from_host(q)
    want = O.canonical_pairs(*O.nested_loop_pairs(q, b))
    assert len(want[0]) >= 1
    assert_all(all_forms(crt, d, rt, dq), want)


def test_query_nan_window_follows_tree_semantics(crt):
    """A NaN coordinate never excludes (src/rtree_bfs_frontier.cuh:40-44): an
    all-NaN window descends everywhere and hits every box; a window with one
    NaN side is bounded by the other three."""
    b = D.uniform_boxes(5_000, seed=53)
    q = D.uniform_windows(20, seed=153)
    for a in (q.xmin, q.ymin, q.xmax, q.ymax):
        a[3] = np.nan
    q.xmin[7] = np.nan
    d, rt, dq, want = setup(crt, b, q, 10)
    assert (want[1] == 3).sum() == b.n
    assert 0 < (want[1] == 7).sum() < b.n
    assert_all(all_forms(crt, d, rt, dq), want)


def boxes_not_ordinary(n, seed):
    """Uniform boxes, 600 of them made not ordinary: inverted in x, a ymax far
    below the ymin, a NaN xmin or a NaN ymax."""
    b = D.uniform_boxes(n, seed=seed)
    k = np.random.default_rng(seed).choice(n, 600, replace=False)
    inv, low, nx, ny = k[:200], k[200:400], k[400:500], k[500:]
    b.xmin[inv], b.xmax[inv] = b.xmax[inv].copy(), b.xmin[inv].copy()
    b.ymax[low] = b.ymin[low] - np.float32(0.02) * D.SCALE
    b.xmin[nx] = np.nan
    b.ymax[ny] = np.nan
    return b


@pytest.mark.parametrize("f", [4, 10, 16])
def test_query_boxes_not_ordinary(crt, f):
    """The predicate (src/rtree_bfs_frontier.cuh:40-44) can reject a box that
    is not ordinary (xmin > xmax, ymin > ymax, or a NaN corner, which the
    MBR's min/max skip) under a node whose MBR the window contains, so such a
    box set must not take the containment shortcut: every form equals the
    oracle's traversal, and the shortcut's test count equals the box-by-box
    one."""
    b = boxes_not_ordinary(80_000, seed=300 + f)
    q = D.mixed_windows(1500, None, seed=400 + f, lo=1e-2, hi=0.5)
    d, rt, dq, want = setup(crt, b, q, f)
    assert len(want[0]) > 100_000
    assert_all(all_forms(crt, d, rt, dq), want)
    for nc in (0, 1):
        got = canon(*crt.query(rt, d, dq, mode=crt.CRT_QUERY_PLAIN, no_contain=nc)[:2])
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), nc
    s = crt.query_stats(rt, d, dq)
    assert s["hits"] == len(want[0]) and s["tested_contain"] == s["tested"]
    assert s["range_hits"] == 0
    # the same boxes made ordinary again: the shortcut is back on
    o = boxes_not_ordinary(80_000, seed=300 + f)
    o.xmin, o.xmax = np.fmin(o.xmin, o.xmax), np.fmax(o.xmin, o.xmax)
    o.ymin, o.ymax = np.fmin(o.ymin, o.ymax), np.fmax(o.ymin, o.ymax)
    d2, rt2, dq2, want2 = setup(crt, o, q, f)
    s2 = crt.query_stats(rt2, d2, dq2)
    assert s2["hits"] == len(want2[0]) and s2["tested_contain"] < s2["tested"]
    got = canon(*crt.query(rt2, d2, dq2))
    assert np.array_equal(got[0], want2[0]) and np.array_equal(got[1], want2[1])


@pytest.mark.parametrize("f", [2, 3, 10, 16, 32, 40])
def test_large_windows_containment(crt, f):
    """Windows covering large parts of the domain: whole subtrees are emitted
    by slot range without per-box tests; the pairs must equal the oracle's and
    those of the box-by-box traversal (no_contain)."""
    b = D.uniform_boxes(150_000, seed=80 + f)
    q = D.mixed_windows(300, b, seed=180 + f, lo=0.05, hi=0.9)
    d, rt, dq, want = setup(crt, b, q, f)
    assert len(want[0]) > 1_000_000
    for mode in (crt.CRT_QUERY_PERSISTENT, crt.CRT_QUERY_PLAIN):
        for nc in (0, 1):
            got = canon(*crt.query(rt, d, dq, mode=mode, no_contain=nc)[:2])
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (mode, nc)
    p = crt.bfs_frontier(rt, d, dq)
    got = canon(*p.to_host())
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_overflow_and_retry(crt):
    import torch
    b = D.uniform_boxes(100_000, seed=54)
    q = D.uniform_windows(3000, seed=154, max_side=0.05)
    d, rt, dq, want = setup(crt, b, q, 10)
    total = len(want[0])
    for mode in (crt.CRT_QUERY_PERSISTENT, crt.CRT_QUERY_PLAIN):
        res = crt.new_result_block()
        cap = 1000
        fid = torch.empty(cap, dtype=torch.int32, device="cuda")
        tid = torch.empty(cap, dtype=torch.int32, device="cuda")
        offs = torch.empty(q.n + 1, dtype=torch.int64, device="cuda") if mode else None
        crt.query_into(rt, d, dq, fid, tid, res, offs, mode)
        r = crt.read_result(res)
        assert r["overflow"] == 1 and r["required"] == total
        cap = crt.query_capacity(r["required"], mode)
        fid = torch.empty(cap, dtype=torch.int32, device="cuda")
        tid = torch.empty(cap, dtype=torch.int32, device="cuda")
        crt.query_into(rt, d, dq, fid, tid, res, offs, mode)
        r = crt.read_result(res)
        assert r["overflow"] == 0 and r["count"] == total
        got = canon(fid[:total], tid[:total])
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_plain_offsets_are_csr(crt):
    b = D.uniform_boxes(50_000, seed=55)
    q = D.uniform_windows(1000, seed=155)
    d, rt, dq, want = setup(crt, b, q, 10)
    fid, tid, offs = crt.query(rt, d, dq, mode=crt.CRT_QUERY_PLAIN)
    offs = offs.cpu().numpy()
    tid = tid.cpu().numpy()
    counts = np.bincount(want[1], minlength=q.n)
    assert np.array_equal(np.diff(offs), counts)
    # grouped by window in window order
    assert np.all(np.diff(tid) >= 0)


def test_plan_graph_replay(crt):
    import torch
    b = D.uniform_boxes(200_000, seed=56)
    q = D.mixed_windows(5000, b, seed=156, lo=1e-4, hi=3e-2)
    d, rt, dq, want = setup(crt, b, q, 10)
    cap = crt.query_capacity(len(want[0]))
    fid = torch.empty(cap, dtype=torch.int32, device="cuda")
    tid = torch.empty(cap, dtype=torch.int32, device="cuda")
    res = crt.new_result_block()
    plan = crt.Plan(rt, d, dq, fid, tid, res)
    for _ in range(3):
        fid.fill_(-1)
        plan.launch()
        r = crt.read_result(res)
        assert r["overflow"] == 0 and r["count"] == len(want[0])
        got = canon(fid[:r["count"]], tid[:r["count"]])
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    plan.destroy()
    # an unsorted plan takes a smaller live window count
    plan = crt.Plan(rt, d, dq, fid, tid, res, sort_windows=0)
    plan.set_nq(1234)
    plan.launch()
    r = crt.read_result(res)
    sel = want[1] < 1234
    got = canon(fid[:r["count"]], tid[:r["count"]])
    assert np.array_equal(got[0], want[0][sel]) and np.array_equal(got[1], want[1][sel])
    plan.destroy()


def test_mixed_windows_clustered_tree_counts(crt):
    """Reduced instance of the uneven-window workload (log-uniform sides up to
    0.1): per-window counts and pair digests equal the oracle's."""
    b = D.clustered_boxes(2_000_000, seed=2, chunk=1_000_000)
    q = D.mixed_windows(20_000, b, seed=157)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(16)
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    sb, t = O.build(b, 16)
    st = O.tree_query_stats(t, sb, q)
    fid, tid = crt.query(rt, d, dq)
    assert fid.numel() == st.total
    gc, gh = O.pair_hashes(fid.cpu().numpy(), tid.cpu().numpy(), q.n)
    assert np.array_equal(gc, st.counts) and np.array_equal(gh, st.hashes)


GOLDEN = [p for p in sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
          if "frontier_fid" in np.load(p)]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_query_matches_reference_golden(crt, path):
    z = np.load(path)
    b = HostBoxes(z["box_xmin"], z["box_ymin"], z["box_xmax"], z["box_ymax"], z["box_id"])
    q = HostBoxes(z["win_xmin"], z["win_ymin"], z["win_xmax"], z["win_ymax"], z["win_id"])
    d = crt.BBox.from_host(b)
    rt = crt.RTree(int(z["fanout"]))
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    want = (z["frontier_fid"], z["frontier_tid"])
    assert_all(all_forms(crt, d, rt, dq), want)


def test_query_stats_match_oracle(crt):
    """Per-window hit counts and leaf boxes tested by the reference's algorithm
    equal the oracle's; the containment traversal tests no more boxes and
    finds the same hits."""
    b = D.clustered_boxes(400_000, seed=11, chunk=400_000)
    q = D.mixed_windows(5_000, b, seed=12)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(16)
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    sb, t = O.build(b, 16)
    want = O.tree_query_stats(t, sb, q)
    st = crt.query_stats(rt, d, dq, per_window=True)
    assert np.array_equal(st["per_window_hits"].cpu().numpy(), want.counts)
    assert np.array_equal(st["per_window_tested"].cpu().numpy(), want.tested)
    assert st["hits"] == int(want.counts.sum())
    assert st["tested"] == int(want.tested.sum())
    assert 0 <= st["tested_contain"] <= st["tested"]
    assert 0 <= st["range_hits"] <= st["hits"]


def test_query_stream_edges(crt):
    """Streamed batches: an empty window set gives no batch and no pairs; a
    window whose own pairs exceed the buffer is CRT_ERR_OUTPUT_OVERFLOW; a
    buffer below the form's chunk slack is rejected."""
    b = D.uniform_boxes(200_000, seed=91)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(16)
    crt.build_rtree(d, rt)
    got = []
    empty = crt.BBox.empty(0)
    st = crt.query_stream(rt, d, empty, lambda f, t, a: got.append(f.numel()),
                          capacity=1 << 20, mode=crt.CRT_QUERY_PLAIN)
    assert st == {"pairs": 0, "batches": 0, "retries": 0} and not got
    # one window over the whole domain: 200k pairs against a 1000-pair buffer
    big = HostBoxes(np.array([-1.0], np.float32), np.array([-1.0], np.float32),
                      np.array([1e9], np.float32), np.array([1e9], np.float32),
                      np.array([0], np.int32))
    dq = crt.BBox.from_host(big)
    with pytest.raises(crt.CrtError):
        crt.query_stream(rt, d, dq, lambda *a: None, capacity=1000, mode=crt.CRT_QUERY_PLAIN)
    with pytest.raises(crt.CrtError):
        crt.query_stream(rt, d, dq, lambda *a: None, capacity=1000)
    # the same window with room: every box once
    ids = []
    st = crt.query_stream(rt, d, dq, lambda f, t, a: ids.append(f.cpu().numpy()),
                          capacity=1 << 20, mode=crt.CRT_QUERY_PLAIN)
    assert st["pairs"] == b.n
    assert np.array_equal(np.sort(np.concatenate(ids)), np.arange(b.n, dtype=np.int32))


def test_plain_csr_without_window_column(crt):
    """Plain form with offsets and no window column: the box ids and offsets
    equal those of the pair output, and the window of every id follows from
    the offsets (CSR).  Without offsets, or in the persistent form, a missing
    window column is rejected."""
    import torch
    b = D.uniform_boxes(300_000, seed=95)
    q = D.mixed_windows(5_000, b, seed=195)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(16)
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    fid, tid, offs = crt.query(rt, d, dq, mode=crt.CRT_QUERY_PLAIN)
    n = fid.numel()
    fid2 = torch.empty(n, dtype=torch.int32, device="cuda")
    offs2 = torch.empty(q.n + 1, dtype=torch.int64, device="cuda")
    res = crt.new_result_block()
    crt.query_into(rt, d, dq, fid2, None, res, offs2, crt.CRT_QUERY_PLAIN)
    r = crt.read_result(res)
    assert r["count"] == n and not r["overflow"] and not r["error"]
    assert torch.equal(offs2, offs) and torch.equal(fid2, fid)
    counts = (offs2[1:] - offs2[:-1]).cpu().numpy()
    tid_from_csr = np.repeat(np.arange(q.n, dtype=np.int32), counts)
    assert np.array_equal(tid_from_csr, tid.cpu().numpy())
    sb, t = O.build(b, 16)
    want = canon(*O.tree_query_pairs(t, sb, q))
    got = canon(fid2.cpu().numpy(), tid_from_csr)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    with pytest.raises(crt.CrtError):
        crt.query_into(rt, d, dq, fid2, None, res, None, crt.CRT_QUERY_PLAIN)
    with pytest.raises(crt.CrtError):
        crt.query_into(rt, d, dq, fid2, None, res, offs2, crt.CRT_QUERY_PERSISTENT)


def test_pairs_digest_matches_oracle(crt):
    """crt_pairs_digest gives the oracle's per-window counts and digests:
    random pairs, a window base offset, pairs outside the window range
    (skipped and counted), and long runs of one window across whole warps
    (the warp-aggregated path), in pieces accumulated call by call."""
    import torch
    rng = np.random.default_rng(11)
    nq = 5000
    parts = []
    # scattered windows, random ids (negative ones included)
    parts.append((rng.integers(-2**31, 2**31, 200_003).astype(np.int32),
                  rng.integers(0, nq, 200_003).astype(np.int32)))
    # long runs: a few windows with 100k+ consecutive pairs each
    runs = np.repeat(np.array([7, 4999, 0, 1234], np.int32), [130_000, 70_001, 4096, 99_999])
    parts.append((rng.integers(-2**31, 2**31, runs.size).astype(np.int32), runs))
    dg = crt.PairDigest(nq)
    want_c = np.zeros(nq, np.int64)
    want_h = np.zeros(nq, np.uint64)
    for fid, tid in parts:
        dg.add(torch.from_numpy(fid).cuda(), torch.from_numpy(tid).cuda())
        c, h = O.pair_hashes(fid, tid, nq)
        want_c += c
        with np.errstate(over="ignore"):
            want_h += h
    # a batch whose window indices are relative to a base; some fall outside
    base = 3000
    fid = rng.integers(-2**31, 2**31, 50_000).astype(np.int32)
    tid = rng.integers(-100, nq - base + 100, 50_000).astype(np.int32)
    dg.add(torch.from_numpy(fid).cuda(), torch.from_numpy(tid).cuda(), window_base=base)
    w = tid.astype(np.int64) + base
    ok = (w >= 0) & (w < nq)
    c, h = O.pair_hashes(fid[ok], w[ok].astype(np.int32), nq)
    want_c += c
    with np.errstate(over="ignore"):
        want_h += h
    gc, gh, bad = dg.to_host()
    assert bad == int((~ok).sum()) and bad > 0
    assert np.array_equal(gc, want_c)
    assert np.array_equal(gh, want_h)


def test_pairs_digest_of_a_query_equals_oracle_stats(crt):
    """The digest of a persistent query's output equals the oracle's tree
    query counts and digests for every window."""
    b = D.clustered_boxes(300_000, seed=17)
    q = D.mixed_windows(20_000, b, seed=117)
    d = crt.BBox.from_host(b)
    rt = crt.RTree(16)
    crt.build_rtree(d, rt)
    dq = crt.BBox.from_host(q)
    fid, tid = crt.query(rt, d, dq)
    dg = crt.PairDigest(q.n)
    dg.add(fid, tid)
    sb, t = O.build(b, 16)
    want = O.tree_query_stats(t, sb, q)
    gc, gh, bad = dg.to_host()
    assert bad == 0 and want.total > 100_000
    assert np.array_equal(gc, want.counts) and np.array_equal(gh, want.hashes)


def test_bad_warps_per_window_is_rejected(crt):
    import torch
    b = D.uniform_boxes(5000, seed=44)
    q = D.uniform_windows(100, seed=144)
    d, rt, dq, want = setup(crt, b, q, 10)
    fid = torch.empty(1 << 16, dtype=torch.int32, device="cuda")
    tid = torch.empty(1 << 16, dtype=torch.int32, device="cuda")
    res = crt.new_result_block()
    with pytest.raises(crt.CrtError):
        crt.query_into(rt, d, dq, fid, tid, res, warps_per_window=3)


@pytest.mark.parametrize("levels", [0, 1, 2, 3, 4, 9])
def test_staging_depths_are_exact(crt, levels):
    """Whole levels staged (as many of `levels` as fit) give the oracle's pairs,
    with windows shared by 1 or 2 warps."""
    b = D.clustered_boxes(400_000, seed=45)
    q = D.mixed_windows(3000, b, seed=145, lo=1e-5, hi=5e-2)
    d, rt, dq, want = setup(crt, b, q, 8)
    for wpw in (1, 2):
        got = canon(*crt.query(rt, d, dq, stage_levels=levels, warps_per_window=wpw))
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), (levels, wpw)
