"""The oracle (CPU restatement) checked against the reference itself: its own
nested_loop_query compiled from source, and golden node arrays / hit pairs
written by its own GPU build and query paths (tests/golden/make_golden.py)."""
import glob
import os

import numpy as np
import pytest

from curtree_b200 import datasets as D
from curtree_b200.datasets import HostBoxes
from oracle import oracle as O


def _bits_equal(a, b):
    """Bitwise float equality, treating any two NaNs as equal."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    if a.shape != b.shape:
        return False
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | both_nan))


def test_dilate_spreads_bits():
    L = O.lib()
    # dilate(v) puts bit k of v at bit 2k (the reference's table, src/z_order.cuh:63-65)
    f = L.orc_dilate16
    f.restype = np.ctypeslib.ctypes.c_uint32
    f.argtypes = [np.ctypeslib.ctypes.c_uint16]
    rng = np.random.default_rng(0)
    for v in list(rng.integers(0, 65536, 200)) + [0, 1, 3, 255, 65535]:
        got = f(int(v))
        want = 0
        for k in range(16):
            want |= ((int(v) >> k) & 1) << (2 * k)
        assert got == want


def test_key_examples():
    # centre (1, 0) -> x bit 0 -> key 1; (0, 1) -> y bit 0 -> key 2; (3, 3) -> 15
    assert O.lib().orc_key(1.0, 0.0, 1.0, 0.0) == 1
    assert O.lib().orc_key(0.0, 1.0, 0.0, 1.0) == 2
    assert O.lib().orc_key(3.0, 3.0, 3.0, 3.0) == 15
    # truncation toward zero of the fp32 centre
    assert O.lib().orc_key(0.0, 0.0, 3.9, 0.0) == O.lib().orc_key(1.0, 0.0, 1.0, 0.0)
    # y >= 2^15 sets bit 31: a negative signed key
    assert O.lib().orc_key(0.0, 40000.0, 0.0, 40000.0) < 0
    # out-of-range centres, as the reference's device build converts them:
    # unsigned 32-bit truncation (saturating), then the low 16 bits
    assert O.lib().orc_f2u16(70000.0) == 70000 & 0xFFFF
    assert O.lib().orc_f2u16(65536.0) == 0
    assert O.lib().orc_f2u16(-5.0) == 0
    assert O.lib().orc_f2u16(float("nan")) == 0
    assert O.lib().orc_f2u16(1e12) == 0xFFFF


def test_sort_is_stable_and_signed():
    k = np.array([5, -1, 5, 0, -1, 2**31 - 1, -(2**31), 5], np.int32)
    p = O.sort_perm(k)
    assert list(p) == [6, 1, 4, 3, 0, 2, 7, 5]
    rng = np.random.default_rng(1)
    k = rng.integers(-50, 50, 10000).astype(np.int32)
    p = O.sort_perm(k)
    assert np.array_equal(p, np.argsort(k, kind="stable"))


def test_levels():
    assert O.levels(1_000_000, 10) == [100000, 10000, 1000, 100, 10, 1]
    assert O.levels(1, 10) == []
    assert O.levels(7, 10) == [1]
    assert O.levels(11, 10) == [2, 1]
    with pytest.raises(ValueError):
        O.levels(0, 10)
    with pytest.raises(ValueError):
        O.levels(10, 1)


def test_level_float_formula_hazard():
    # the reference's ceil((float)len/d) agrees with the exact ceiling at every
    # workload size used here ...
    for n in (1_000_000, 2_000_000, 5_000_000, 10_000_000, 20_000_000, 50_000_000, 100_000_000):
        for f in (8, 10, 16, 32):
            assert O.levels(n, f) == O.levels(n, f, ref_float=True)
    # ... but not for every n above 2^24
    bad = [n for n in range(2**24 + 1, 2**24 + 400) if O.levels(n, 10) != O.levels(n, 10, ref_float=True)]
    assert bad, "expected sizes where the float formula departs from the exact ceiling"


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_tree_query_equals_brute_force(seed):
    b = D.uniform_boxes(30000, seed=seed)
    q = D.mixed_windows(300, b, seed=100 + seed, lo=1e-4, hi=3e-2)
    for f in (3, 10, 33):
        sb, t = O.build(b, f)
        st = O.tree_query_stats(t, sb, q)
        c, h = O.nested_loop_stats(q, b)
        assert np.array_equal(st.counts, c)
        assert np.array_equal(st.hashes, h)
    fid, tid = O.tree_query_pairs(t, sb, q)
    did, qid = O.nested_loop_pairs(q, b)
    f2, t2 = O.canonical_pairs(fid, tid)
    assert np.array_equal(f2, did) and np.array_equal(t2, qid)


def test_build_structure():
    b = D.uniform_boxes(12345, seed=4)
    sb, t = O.build(b, 10)
    lv = O.levels(b.n, 10)
    assert t.sz == sum(lv)
    # root first, levels downward; children contiguous; leaf-parents point at slots
    rsz = t.sz
    start = rsz - lv[0]
    assert np.all(t.pos[start:] == rsz + 10 * np.arange(lv[0]))
    assert t.len[start:].sum() == b.n
    # every box lies inside its leaf-parent
    node_of_slot = start + np.arange(b.n) // 10
    assert np.all(sb.xmin >= t.xmin[node_of_slot]) and np.all(sb.xmax <= t.xmax[node_of_slot])
    # the sorted ids are a permutation
    assert np.array_equal(np.sort(sb.id), np.arange(b.n))


def test_raw_unit_data_degenerates():
    b = D.uniform_boxes(5000, seed=3, scale=False)
    assert np.all(O.keys(b) == 0)
    sb, t = O.build(b, 10)
    assert np.array_equal(sb.id, np.arange(b.n))  # identity order


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
@pytest.mark.parametrize("maker", ["uniform", "touching", "specials"])
def test_brute_force_matches_reference_nested_loop(maker):
    if maker == "uniform":
        b = D.uniform_boxes(20000, seed=5)
        q = D.uniform_windows(300, seed=105)
    elif maker == "touching":
        b = D.uniform_boxes(5000, seed=6)
        q = b.take(np.arange(0, 5000, 50))
        q.id = np.arange(q.n, dtype=np.int32)
    else:
        rng = np.random.default_rng(8)
        cx = rng.uniform(-100, 70000, 3000)
        cy = rng.uniform(-100, 70000, 3000)
        w = rng.uniform(0, 300, 3000)
        w[::5] = 0
        b = HostBoxes(*(np.asarray(a, np.float32) for a in (cx - w, cy - w, cx + w, cy + w)),
                      np.arange(3000, dtype=np.int32))
        q = b.take(np.arange(0, 3000, 30))
        q.id = np.arange(q.n, dtype=np.int32)
    rd, rq = O.ref_nested_loop_pairs(q, b)
    od, oq = O.nested_loop_pairs(q, b)
    assert np.array_equal(rd, od) and np.array_equal(rq, oq)
    assert len(rd) > 0


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _golden_boxes(z, prefix):
    return HostBoxes(z[prefix + "xmin"], z[prefix + "ymin"], z[prefix + "xmax"], z[prefix + "ymax"],
                     z[prefix + "id"])


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 10, "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_build_matches_reference_golden(path):
    z = np.load(path)
    b = _golden_boxes(z, "box_")
    f = int(z["fanout"])
    sb, t = O.build(b, f)
    assert np.array_equal(sb.id, z["sorted_id"])
    for k in ("xmin", "ymin", "xmax", "ymax"):
        assert _bits_equal(getattr(t, k), z["node_" + k]), k
    assert np.array_equal(t.pos, z["node_pos"])
    assert np.array_equal(t.len, z["node_len"])


@pytest.mark.parametrize("path", [p for p in GOLDEN if "frontier_fid" in np.load(p)],
                         ids=[os.path.basename(p) for p in GOLDEN if "frontier_fid" in np.load(p)])
def test_oracle_query_matches_reference_golden(path):
    z = np.load(path)
    b = _golden_boxes(z, "box_")
    q = _golden_boxes(z, "win_")
    sb, t = O.build(b, int(z["fanout"]))
    fid, tid = O.canonical_pairs(*O.tree_query_pairs(t, sb, q))
    assert np.array_equal(fid, z["frontier_fid"]) and np.array_equal(tid, z["frontier_tid"])
    if "thrust_fid" in z:
        assert np.array_equal(fid, z["thrust_fid"]) and np.array_equal(tid, z["thrust_tid"])
    # and the brute force agrees (no NaN in query fixtures)
    did, qid = O.nested_loop_pairs(q, b)
    assert np.array_equal(fid, did) and np.array_equal(tid, qid)


def test_quadratic_rtree_matches_brute_force():
    """The CPU R-tree of the reference's Boost check, restated (Guttman's
    quadratic split, 4-16 entries per node, built by insertion): every
    window's pair count and digest equal the brute force's, on uniform and
    clustered boxes with duplicates and points, with window ids."""
    from curtree_b200 import datasets as D
    for b in (D.uniform_boxes(60_000, seed=31), D.clustered_boxes(60_000, seed=32, chunk=60_000)):
        q = D.mixed_windows(3000, b, seed=131)
        t = O.QuadraticRTree(b)
        ids = np.arange(5, 5 + q.n, dtype=np.int32)
        c, h, _ = t.query_stats(q, qid=ids, nthreads=4)
        t.free()
        fid, qo = O.nested_loop_pairs(q, b)
        wc, wh = O.pair_hashes(fid, ids[qo], 5 + q.n)
        assert c.sum() > 10_000
        assert np.array_equal(c, wc[5:]) and np.array_equal(h, wh[5:])
