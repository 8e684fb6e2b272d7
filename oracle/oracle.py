"""Python view of the CPU oracle (oracle/crt_oracle.c) and of the reference's
own CPU brute force compiled from its sources (oracle/_ref/libref_cpu.so).

TEST INFRASTRUCTURE ONLY.  The test suite, the smoke check and the benchmark's
CPU-baseline leg import this module as the checker; the product library never
does, and it has no CPU fallback through it.

Each wrapper names the reference code it restates; the C file carries the
file:line citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF_CPU = os.path.join(HERE, "_ref", "libref_cpu.so")
_lib = None
_ref = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64


def build() -> None:
    """Compile liboracle.so (and the reference CPU/GPU runners when the
    reference sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.orc_key.restype = ctypes.c_int32
        L.orc_key.argtypes = [ctypes.c_float] * 4
        L.orc_f2u16.restype = ctypes.c_uint16
        L.orc_f2u16.argtypes = [ctypes.c_float]
        L.orc_keys.argtypes = [_f32p, _f32p, _f32p, _f32p, _i64, _i32p]
        L.orc_sort_perm.restype = ctypes.c_int
        L.orc_sort_perm.argtypes = [_i32p, _i64, _i32p]
        L.orc_levels.restype = ctypes.c_int
        L.orc_levels.argtypes = [_i64, ctypes.c_int, _i64p, ctypes.c_int]
        L.orc_levels_ref_float.restype = ctypes.c_int
        L.orc_levels_ref_float.argtypes = [_i64, ctypes.c_int, _i64p, ctypes.c_int]
        L.orc_build.restype = _i64
        L.orc_build.argtypes = [_f32p] * 4 + [_i32p, _i64, ctypes.c_int] + [_f32p] * 4 + [_i32p] + \
            [_f32p] * 4 + [_i32p, _i32p]
        tree_args = [_f32p] * 4 + [_i32p, _i32p, _i64, ctypes.c_int] + [_f32p] * 4 + [_i32p, _i64] + \
            [_f32p] * 4 + [_i64]
        L.orc_tree_query_stats.restype = ctypes.c_int
        L.orc_tree_query_stats.argtypes = tree_args + [_i64p, _u64p, _i64p, _i64p, ctypes.c_int]
        L.orc_tree_query_stats_ids.restype = ctypes.c_int
        L.orc_tree_query_stats_ids.argtypes = tree_args[:-1] + [_i32p, _i64] + \
            [_i64p, _u64p, _i64p, _i64p, ctypes.c_int]
        L.orc_tree_query_pairs.restype = _i64
        L.orc_tree_query_pairs.argtypes = tree_args + [_i32p, _i32p, _i64]
        nl_args = [_f32p] * 4 + [_i32p, _i64] + [_f32p] * 4 + [_i32p, _i64]
        L.orc_nested_loop_stats.restype = ctypes.c_int
        L.orc_nested_loop_stats.argtypes = nl_args + [_i64p, _u64p, ctypes.c_int]
        L.orc_nested_loop_pairs.restype = _i64
        L.orc_nested_loop_pairs.argtypes = nl_args + [_i32p, _i32p, _i64]
        L.orc_qrtree_build.restype = ctypes.c_void_p
        L.orc_qrtree_build.argtypes = [_f32p] * 4 + [_i32p, _i64, ctypes.POINTER(ctypes.c_double)]
        L.orc_qrtree_free.restype = None
        L.orc_qrtree_free.argtypes = [ctypes.c_void_p]
        L.orc_qrtree_query_stats.restype = ctypes.c_int
        L.orc_qrtree_query_stats.argtypes = [ctypes.c_void_p] + [_f32p] * 4 + [ctypes.c_void_p, _i64,
                                                                                _i64p, _u64p, ctypes.c_int,
                                                                                ctypes.POINTER(ctypes.c_double)]
        L.orc_pair_hash.restype = ctypes.c_uint64
        L.orc_pair_hash.argtypes = [ctypes.c_int32, ctypes.c_int32]
        _lib = L
    return _lib


def ref_cpu_available() -> bool:
    return os.path.exists(_REF_CPU)


def ref_cpu():
    """The reference's nested_loop_query (src/utility.h:22-45) compiled from its
    sources by `make -C oracle ref`."""
    global _ref
    if _ref is None:
        R = ctypes.CDLL(_REF_CPU)
        args = [_f32p] * 4 + [_i32p, ctypes.c_int] + [_f32p] * 4 + [_i32p, ctypes.c_int]
        R.ref_nested_loop_query.restype = _i64
        R.ref_nested_loop_query.argtypes = args + [_i32p, _i32p, _i64]
        R.ref_nested_loop_query_mt.restype = _i64
        R.ref_nested_loop_query_mt.argtypes = args + [ctypes.c_int]
        R.ref_nested_loop_query_mt_digest.restype = _i64
        R.ref_nested_loop_query_mt_digest.argtypes = args + [ctypes.c_int, _i64p, _u64p,
                                                             ctypes.POINTER(ctypes.c_double)]
        R.ref_read_mbr.restype = ctypes.c_int
        R.ref_read_mbr.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_float] + [_f32p] * 4 + [_i32p]
        _ref = R
    return _ref


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _box_args(b):
    return [_c(b.xmin, np.float32), _c(b.ymin, np.float32), _c(b.xmax, np.float32),
            _c(b.ymax, np.float32)]


@dataclass
class HostTree:
    """Node arrays in the reference's RTREE<float> layout (src/rtree.h:13-23)."""

    xmin: np.ndarray
    ymin: np.ndarray
    xmax: np.ndarray
    ymax: np.ndarray
    pos: np.ndarray
    len: np.ndarray
    fanout: int

    @property
    def sz(self) -> int:
        return int(self.xmin.shape[0])


def keys(boxes) -> np.ndarray:
    """mbr2key of every box (src/rtree_bulkload_thrust.cuh:52-60), as int32."""
    out = np.empty(boxes.n, np.int32)
    lib().orc_keys(*_box_args(boxes), boxes.n, out)
    return out


def sort_perm(k: np.ndarray) -> np.ndarray:
    """Stable sort positions by signed key (src/rtree_bulkload_thrust.cuh:83-86)."""
    k = _c(k, np.int32)
    perm = np.empty(k.shape[0], np.int32)
    if lib().orc_sort_perm(k, k.shape[0], perm) != 0:
        raise MemoryError("oracle sort")
    return perm


def levels(n: int, fanout: int, ref_float: bool = False) -> list[int]:
    """Node count per level, leaf-parents first (src/rtree_bulkload_thrust.cuh:103-115)."""
    buf = np.zeros(64, np.int64)
    fn = lib().orc_levels_ref_float if ref_float else lib().orc_levels
    m = fn(n, fanout, buf, 64)
    if m < 0:
        raise ValueError(f"no tree for n={n}, fanout={fanout}")
    return [int(x) for x in buf[:m]]


def build(boxes, fanout: int):
    """build_rtree (src/rtree_bulkload_thrust.cuh:62-213): returns the boxes in
    sorted slot order and the node arrays."""
    from curtree_b200.datasets import HostBoxes

    n = boxes.n
    lv = levels(n, fanout)
    rsz = sum(lv)
    sb = HostBoxes(np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32),
                   np.empty(n, np.float32), np.empty(n, np.int32))
    t = HostTree(np.empty(rsz, np.float32), np.empty(rsz, np.float32), np.empty(rsz, np.float32),
                 np.empty(rsz, np.float32), np.empty(rsz, np.int32), np.empty(rsz, np.int32), fanout)
    # zero-length arrays still need a valid pointer
    if rsz == 0:
        t = HostTree(*(np.empty(1, d) for d in [np.float32] * 4 + [np.int32] * 2), fanout)
    got = lib().orc_build(*_box_args(boxes), _c(boxes.id, np.int32), n, fanout,
                          sb.xmin, sb.ymin, sb.xmax, sb.ymax, sb.id,
                          t.xmin, t.ymin, t.xmax, t.ymax, t.pos, t.len)
    if got < 0:
        raise ValueError(f"oracle build failed ({got})")
    if rsz == 0:
        t = HostTree(*(a[:0] for a in (t.xmin, t.ymin, t.xmax, t.ymax, t.pos, t.len)), fanout)
    return sb, t


def _tree_args(tree: HostTree, sboxes, q):
    def nz(a, dt):
        a = _c(a, dt)
        return a if a.size else np.zeros(1, dt)
    return [nz(tree.xmin, np.float32), nz(tree.ymin, np.float32), nz(tree.xmax, np.float32),
            nz(tree.ymax, np.float32), nz(tree.pos, np.int32), nz(tree.len, np.int32), tree.sz,
            tree.fanout] + [nz(a, np.float32) for a in (sboxes.xmin, sboxes.ymin, sboxes.xmax,
                                                        sboxes.ymax)] + \
        [nz(sboxes.id, np.int32), sboxes.n] + [nz(a, np.float32) for a in (q.xmin, q.ymin,
                                                                           q.xmax, q.ymax)] + [q.n]


@dataclass
class QueryStats:
    counts: np.ndarray   # hits per query
    hashes: np.ndarray   # order-independent digest of each query's hit pairs
    tested: np.ndarray   # leaf boxes tested per query (T_leaf)
    visited: np.ndarray  # node MBR tests per query

    @property
    def total(self) -> int:
        return int(self.counts.sum())


def tree_query_stats(tree: HostTree, sboxes, q, nthreads: int | None = None,
                     qid: np.ndarray | None = None) -> QueryStats:
    """Per-query counts/digests of the reference's tree query semantics
    (src/rtree_bfs_frontier.cuh:60-289, src/rtree_bfs_thrust.cuh:95-250).
    qid: the windows' indices used in the digests (default: positional)."""
    nthreads = nthreads or os.cpu_count() or 1
    nq = max(q.n, 1)
    st = QueryStats(np.zeros(nq, np.int64), np.zeros(nq, np.uint64), np.zeros(nq, np.int64),
                    np.zeros(nq, np.int64))
    if qid is None:
        rc = lib().orc_tree_query_stats(*_tree_args(tree, sboxes, q), st.counts, st.hashes,
                                        st.tested, st.visited, nthreads)
    else:
        a = _tree_args(tree, sboxes, q)
        ids = _c(qid, np.int32) if q.n else np.zeros(1, np.int32)
        rc = lib().orc_tree_query_stats_ids(*a[:-1], ids, a[-1], st.counts, st.hashes, st.tested,
                                            st.visited, nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle tree query failed ({rc})")
    if q.n == 0:
        st = QueryStats(*(a[:0] for a in (st.counts, st.hashes, st.tested, st.visited)))
    return st


def tree_query_pairs(tree: HostTree, sboxes, q) -> tuple[np.ndarray, np.ndarray]:
    """All hit pairs (fid = box id, tid = query index) of the tree query."""
    n = lib().orc_tree_query_pairs(*_tree_args(tree, sboxes, q), np.zeros(1, np.int32),
                                   np.zeros(1, np.int32), 0)
    if n < 0:
        raise RuntimeError(f"oracle tree query failed ({n})")
    fid = np.empty(max(n, 1), np.int32)
    tid = np.empty(max(n, 1), np.int32)
    lib().orc_tree_query_pairs(*_tree_args(tree, sboxes, q), fid, tid, n)
    return fid[:n], tid[:n]


def nested_loop_stats(q, d, nthreads: int | None = None, positional_qid: bool = True):
    """Per-query counts/digests of the brute force (src/utility.h:22-45)."""
    nthreads = nthreads or os.cpu_count() or 1
    nq = max(q.n, 1)
    counts = np.zeros(nq, np.int64)
    hashes = np.zeros(nq, np.uint64)
    qid = np.arange(q.n, dtype=np.int32) if positional_qid else _c(q.id, np.int32)
    lib().orc_nested_loop_stats(*_box_args(q), qid if q.n else np.zeros(1, np.int32), q.n,
                                *_box_args(d), _c(d.id, np.int32), d.n, counts, hashes, nthreads)
    return counts[:q.n], hashes[:q.n]


def nested_loop_pairs(q, d, positional_qid: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """Brute-force pairs (did, qid) in the reference's order: queries ascending,
    then data in input order (src/utility.h:25-43)."""
    qid = np.arange(q.n, dtype=np.int32) if positional_qid else _c(q.id, np.int32)
    args = [*_box_args(q), qid, q.n, *_box_args(d), _c(d.id, np.int32), d.n]
    n = lib().orc_nested_loop_pairs(*args, np.zeros(1, np.int32), np.zeros(1, np.int32), 0)
    did = np.empty(max(n, 1), np.int32)
    qo = np.empty(max(n, 1), np.int32)
    lib().orc_nested_loop_pairs(*args, did, qo, n)
    return did[:n], qo[:n]


def ref_nested_loop_pairs(q, d, positional_qid: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """The reference's own nested_loop_query, run unchanged on the host."""
    R = ref_cpu()
    qid = np.arange(q.n, dtype=np.int32) if positional_qid else _c(q.id, np.int32)
    args = [*_box_args(q), qid, q.n, *_box_args(d), _c(d.id, np.int32), d.n]
    n = R.ref_nested_loop_query(*args, np.zeros(1, np.int32), np.zeros(1, np.int32), 0)
    did = np.empty(max(n, 1), np.int32)
    qo = np.empty(max(n, 1), np.int32)
    R.ref_nested_loop_query(*args, did, qo, n)
    return did[:n], qo[:n]


def ref_nested_loop_digest(q, d, qid, nthreads: int | None = None):
    """The reference's own nested_loop_query over window slices on host
    threads, with each window's pair count and digest taken from the pairs
    it emitted (qid = the windows' indices, used as the digest's window).
    Returns (counts, hashes, pairs, seconds of the nested_loop_query calls)."""
    nthreads = nthreads or os.cpu_count() or 1
    counts = np.zeros(max(q.n, 1), np.int64)
    hashes = np.zeros(max(q.n, 1), np.uint64)
    secs = ctypes.c_double(0)
    n = ref_cpu().ref_nested_loop_query_mt_digest(*_box_args(q), _c(qid, np.int32), q.n,
                                                  *_box_args(d), _c(d.id, np.int32), d.n,
                                                  nthreads, counts, hashes, ctypes.byref(secs))
    return counts[:q.n], hashes[:q.n], int(n), secs.value


class QuadraticRTree:
    """The reference's CPU check's index (src/verify.hpp:35-95: Boost's
    rtree<value, quadratic<16>>, built by inserting the boxes one at a time),
    restated: Guttman's R-tree with the quadratic split, 4-16 entries per
    node (orc_qrtree_* in crt_oracle.c).  Boost is not available here."""

    def __init__(self, boxes):
        secs = ctypes.c_double(0)
        self._keep = [_c(a, np.float32) for a in (boxes.xmin, boxes.ymin, boxes.xmax, boxes.ymax)]
        self._id = _c(boxes.id, np.int32)
        self.h = lib().orc_qrtree_build(*self._keep, self._id, boxes.n, ctypes.byref(secs))
        if not self.h:
            raise MemoryError("quadratic R-tree build failed")
        self.build_seconds = secs.value

    def query_stats(self, q, qid=None, nthreads: int | None = None):
        """(counts, digests, seconds of the queries) for the windows q."""
        nthreads = nthreads or os.cpu_count() or 1
        counts = np.zeros(max(q.n, 1), np.int64)
        hashes = np.zeros(max(q.n, 1), np.uint64)
        ids = _c(qid, np.int32) if qid is not None else None
        secs = ctypes.c_double(0)
        rc = lib().orc_qrtree_query_stats(self.h, *_box_args(q),
                                          ids.ctypes.data if ids is not None else None, q.n,
                                          counts, hashes, nthreads, ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError(f"quadratic R-tree query failed ({rc})")
        return counts[:q.n], hashes[:q.n], secs.value

    def free(self):
        if self.h:
            lib().orc_qrtree_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def ref_read_mbr(path: str, n: int, r: float):
    """The reference's own readMBR (src/utility.cpp:5-40) on an existing file."""
    from curtree_b200.datasets import HostBoxes
    out = HostBoxes(*(np.empty(n, np.float32) for _ in range(4)), np.empty(n, np.int32))
    rc = ref_cpu().ref_read_mbr(path.encode(), n, r, out.xmin, out.ymin, out.xmax, out.ymax, out.id)
    if rc != 0:
        raise ValueError("reference readMBR rejected the file")
    return out


def canonical_pairs(fid: np.ndarray, tid: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Pairs sorted by (query, box id): the order the reference's drivers
    produce with two stable sorts (src/rtree_test_frontier.cu:102-105)."""
    fid = np.asarray(fid, np.int32)
    tid = np.asarray(tid, np.int32)
    o = np.lexsort((fid, tid))
    return fid[o], tid[o]


def pair_hashes(fid: np.ndarray, tid: np.ndarray, nq: int) -> tuple[np.ndarray, np.ndarray]:
    """Per-query counts and digests of a pair list, with the oracle's digest."""
    fid = np.asarray(fid, np.int64) & 0xFFFFFFFF
    tid = np.asarray(tid, np.int64)
    z = ((tid.astype(np.uint64) & np.uint64(0xFFFFFFFF)) << np.uint64(32)) | fid.astype(np.uint64)
    h = mix64(z)
    counts = np.bincount(tid, minlength=nq).astype(np.int64)
    hashes = np.zeros(nq, np.uint64)
    np.add.at(hashes, tid, h)
    return counts, hashes


def mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser, the per-pair digest of orc_pair_hash."""
    with np.errstate(over="ignore"):
        z = z.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))
