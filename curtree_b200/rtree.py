"""Host-side mirror of the reference's R-tree interface over the crtree C ABI.

The names, argument meaning and ownership follow trxcllnt/curtree:
  build_rtree(d_box, d_rt)              src/rtree_bulkload_thrust.cuh:62-213
  bfs_frontier(d_rt, d_rbox, d_qbox)    src/rtree_bfs_frontier.cuh:292-529
  bfs_thrust(d_rt, d_rbox, d_qbox)      src/rtree_bfs_thrust.cuh:59-256
  BBox / RTree / IDPair                 src/rtree.h:3-29
with the reference's failure modes turned into exceptions (CrtError) instead
of exit()/assert.  Device memory for inputs is allocated through PyTorch
(plumbing only); node arrays and pair arrays returned by build/query are
allocated by the library with cudaMalloc, exactly as the reference's
rt_d_alloc / idpair_d_alloc do, and are released with free().

Extended API: query_into (caller-owned output, int64 counts,
overflow-and-retry, plain or persistent form) and Plan (a persistent query
recorded as a CUDA graph).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, load
from .datasets import HostBoxes

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _stream_handle(stream=None):
    if stream is None:
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class _DeviceBytes:
    """A raw device byte range, seen by torch through the CUDA array
    interface (no copy)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 2}


def _device_bytes(ptr: int, nbytes: int):
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device="cuda")


def _d2h(ptr: int, n: int, dtype) -> np.ndarray:
    """Copy n elements at a device address into a new numpy array."""
    out = np.empty(n, dtype)
    if n:
        out[:] = _device_bytes(ptr, n * out.itemsize).cpu().numpy().view(dtype)
    return out


def _copy_ptr(dst: int, src: int, nbytes: int) -> None:
    """Device-to-device copy between raw addresses on the current stream."""
    if nbytes:
        _device_bytes(dst, nbytes).copy_(_device_bytes(src, nbytes))
        torch.cuda.current_stream().synchronize()


class BBox:
    """Device box set in BBOX<float> layout; the arrays are torch CUDA tensors."""

    def __init__(self, xmin, ymin, xmax, ymax, id):
        self.xmin, self.ymin, self.xmax, self.ymax, self.id = xmin, ymin, xmax, ymax, id

    @property
    def sz(self) -> int:
        return int(self.xmin.numel())

    @classmethod
    def from_host(cls, hb: HostBoxes, device: str = "cuda") -> "BBox":
        f = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(device)
        return cls(f(hb.xmin, np.float32), f(hb.ymin, np.float32), f(hb.xmax, np.float32),
                   f(hb.ymax, np.float32), f(hb.id, np.int32))

    @classmethod
    def empty(cls, n: int, device: str = "cuda") -> "BBox":
        e = lambda dt: torch.empty(n, dtype=dt, device=device)
        return cls(e(torch.float32), e(torch.float32), e(torch.float32), e(torch.float32),
                   e(torch.int32))

    def c(self) -> _lib.crt_bbox_f32:
        return _lib.crt_bbox_f32(self.sz, self.xmin.data_ptr(), self.ymin.data_ptr(),
                                 self.xmax.data_ptr(), self.ymax.data_ptr(), self.id.data_ptr())

    def to_host(self) -> HostBoxes:
        g = lambda t: t.cpu().numpy()
        return HostBoxes(g(self.xmin), g(self.ymin), g(self.xmax), g(self.ymax), g(self.id))


class RTree:
    """Node arrays in RTREE<float> layout.  `owned` trees were allocated by
    build_rtree (library cudaMalloc) and are released by free(); trees built
    with build_into wrap torch tensors."""

    def __init__(self, fanout: int):
        self.s = _lib.crt_rtree_f32(0, fanout, None, None, None, None, None, None)
        self.owned = False
        self._tensors = None

    @property
    def sz(self) -> int:
        return int(self.s.sz)

    @property
    def fanout(self) -> int:
        return int(self.s.fanout)

    def c(self) -> _lib.crt_rtree_f32:
        return self.s

    def to_host(self):
        from types import SimpleNamespace
        n = self.sz
        g = lambda p, dt: _d2h(p, n, dt) if n else np.empty(0, dt)
        return SimpleNamespace(xmin=g(self.s.xmin, np.float32), ymin=g(self.s.ymin, np.float32),
                               xmax=g(self.s.xmax, np.float32), ymax=g(self.s.ymax, np.float32),
                               pos=g(self.s.pos, np.int32), len=g(self.s.len, np.int32),
                               fanout=self.fanout, sz=n)

    def free(self) -> None:
        if self.owned:
            check(load().crt_rtree_free(ctypes.byref(self.s)), "crt_rtree_free")
            self.owned = False
        self._tensors = None
        self.s.sz = 0

    def __del__(self):
        try:
            if self.owned and _lib._lib is not None:
                self.free()
        except Exception:
            pass


class IDPair:
    """Hit pairs in IDPAIR layout (fid = box id, tid = window index),
    allocated by the library; release with free()."""

    def __init__(self):
        self.s = _lib.crt_idpair(0, None, None)

    @property
    def sz(self) -> int:
        return int(self.s.sz)

    def to_host(self):
        return _d2h(self.s.fid, self.sz, np.int32), _d2h(self.s.tid, self.sz, np.int32)

    def free(self) -> None:
        check(load().crt_idpair_free(ctypes.byref(self.s)), "crt_idpair_free")
        self.s.sz = 0

    def __del__(self):
        try:
            if self.s.fid and _lib._lib is not None:
                self.free()
        except Exception:
            pass


def tree_size(n: int, fanout: int) -> int:
    return int(load().crt_tree_size(n, fanout))


def build_rtree(d_box: BBox, d_rt: RTree, stream=None) -> int:
    """build_rtree: sorts d_box in place into Z-order, allocates and fills the
    node arrays of d_rt (fanout read from d_rt), returns R_sz."""
    c = d_box.c()
    rsz = ctypes.c_int32(0)
    st = load().crt_build_f32(ctypes.byref(c), ctypes.byref(d_rt.s), _stream_handle(stream),
                              ctypes.byref(rsz))
    check(st, "build_rtree")
    d_rt.owned = d_rt.s.sz > 0
    return int(rsz.value)


def build_into(d_in: BBox, fanout: int, stream=None) -> tuple[BBox, RTree]:
    """Out-of-place build into torch-allocated arrays."""
    n = d_in.sz
    rsz = tree_size(n, fanout)
    if rsz < 0:
        raise _lib.CrtError(_lib.CRT_ERR_INVALID_ARG, "build_into")
    out = BBox.empty(n)
    rt = RTree(fanout)
    ts = [torch.empty(max(rsz, 1), dtype=dt, device="cuda")
          for dt in [torch.float32] * 4 + [torch.int32] * 2]
    rt.s.xmin, rt.s.ymin, rt.s.xmax, rt.s.ymax, rt.s.pos, rt.s.len = [t.data_ptr() for t in ts]
    rt._tensors = ts
    ci, co = d_in.c(), out.c()
    check(load().crt_build_into_f32(ctypes.byref(ci), ctypes.byref(co), ctypes.byref(rt.s),
                                    _stream_handle(stream)), "build_into")
    return out, rt


def _query_dropin(fn, name, d_rt, d_rbox, d_qbox, stream):
    out = IDPair()
    rb, qb = d_rbox.c(), d_qbox.c()
    check(fn(ctypes.byref(d_rt.s), ctypes.byref(rb), ctypes.byref(qb), ctypes.byref(out.s),
             _stream_handle(stream)), name)
    return out


def bfs_frontier(d_rt: RTree, d_rbox: BBox, d_qbox: BBox, stream=None) -> IDPair:
    """Every (box id, window index) pair whose boxes intersect."""
    return _query_dropin(load().crt_query_f32, "bfs_frontier", d_rt, d_rbox, d_qbox, stream)


def bfs_thrust(d_rt: RTree, d_rbox: BBox, d_qbox: BBox, stream=None) -> IDPair:
    """Same pair set as bfs_frontier (the reference's second query path)."""
    return _query_dropin(load().crt_query_thrust_f32, "bfs_thrust", d_rt, d_rbox, d_qbox, stream)


def canonicalize(fid, tid, stream=None) -> None:
    """Sort pair tensors in place into (window, box id) order on the GPU."""
    n = int(fid.numel())
    check(load().crt_pairs_canonicalize(fid.data_ptr() if n else None,
                                        tid.data_ptr() if n else None, n,
                                        _stream_handle(stream)), "canonicalize")


class PairDigest:
    """Per-window pair counts and order-independent digests accumulated on
    the device (crt_pairs_digest): int64 counts and uint64 digests (held in
    an int64 tensor) for nq windows, plus a count of pairs whose window index
    fell outside [0, nq)."""

    def __init__(self, nq: int):
        self.nq = int(nq)
        self.counts = torch.zeros(max(self.nq, 1), dtype=torch.int64, device="cuda")
        self.hashes = torch.zeros(max(self.nq, 1), dtype=torch.int64, device="cuda")
        self.bad = torch.zeros(1, dtype=torch.int64, device="cuda")

    def add_ptr(self, fid_ptr: int, tid_ptr: int, n: int, window_base: int = 0, stream=None):
        if n <= 0:
            return
        check(load().crt_pairs_digest(fid_ptr, tid_ptr, int(n), int(window_base), self.nq,
                                      self.counts.data_ptr(), self.hashes.data_ptr(),
                                      self.bad.data_ptr(), _stream_handle(stream)),
              "pairs_digest")

    def add(self, fid, tid, window_base: int = 0, n: int | None = None, stream=None):
        n = int(fid.numel()) if n is None else int(n)
        if n:
            self.add_ptr(fid.data_ptr(), tid.data_ptr(), n, window_base, stream)

    def to_host(self) -> tuple[np.ndarray, np.ndarray, int]:
        """(counts int64, digests uint64, pairs outside the window range)."""
        c = self.counts.cpu().numpy()[:self.nq]
        h = self.hashes.cpu().numpy().view(np.uint64)[:self.nq]
        return c, h, int(self.bad.item())


def query_capacity(pairs: int, mode: int = _lib.CRT_QUERY_PERSISTENT, **opts) -> int:
    """Output slots for `pairs` pairs in this mode (persistent: plus the
    per-warp chunk slack of the options' chunk)."""
    o = _lib.default_opts(mode=mode, **opts)
    return int(load().crt_query_capacity(pairs, ctypes.byref(o)))


def query_into(d_rt: RTree, d_rbox: BBox, d_qbox: BBox, fid, tid, result, offsets=None,
               mode: int = _lib.CRT_QUERY_PERSISTENT, stream=None, **opts) -> None:
    """Asynchronous extended query into caller-owned torch tensors: fid/tid
    (int32, capacity = numel), result (uint8 x 64 on the device, the
    crt_query_result block), offsets (int64, nq + 1, plain mode only).  In
    plain mode with offsets, tid may be None: the output is then CSR (box
    ids of window w at fid[offsets[w]:offsets[w + 1]])."""
    o = _lib.default_opts(mode=mode, **opts)
    rb, qb = d_rbox.c(), d_qbox.c()
    cap = int(fid.numel())
    check(load().crt_query_into_f32(ctypes.byref(d_rt.s), ctypes.byref(rb), ctypes.byref(qb),
                                    fid.data_ptr() if cap else None,
                                    tid.data_ptr() if (cap and tid is not None) else None, cap,
                                    result.data_ptr(),
                                    offsets.data_ptr() if offsets is not None else None,
                                    ctypes.byref(o), _stream_handle(stream)), "query_into")


def read_result(result) -> dict:
    """Decode a crt_query_result block held in a torch uint8 tensor."""
    raw = result.cpu().numpy().tobytes()
    r = _lib.crt_query_result.from_buffer_copy(raw)
    return {"count": int(r.count), "required": int(r.required), "overflow": int(r.overflow),
            "error": int(r.error)}


def new_result_block():
    return torch.zeros(64, dtype=torch.uint8, device="cuda")


def query(d_rt: RTree, d_rbox: BBox, d_qbox: BBox, mode: int = _lib.CRT_QUERY_PERSISTENT,
          capacity: int | None = None, stream=None, **opts):
    """Synchronous extended query with overflow-and-retry; returns
    (fid, tid) torch tensors of exactly `count` pairs (and offsets in plain mode)."""
    res = new_result_block()
    chunk = {"chunk": opts["chunk"]} if "chunk" in opts else {}
    cap = capacity if capacity is not None else query_capacity(max(64 * d_qbox.sz, 1024), mode,
                                                               **chunk)
    nq = d_qbox.sz
    for _ in range(3):
        fid = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        tid = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        offs = torch.empty(nq + 1, dtype=torch.int64, device="cuda") \
            if mode == _lib.CRT_QUERY_PLAIN else None
        query_into(d_rt, d_rbox, d_qbox, fid[:cap], tid[:cap], res, offs, mode, stream, **opts)
        r = read_result(res)
        if r["error"]:
            raise _lib.CrtError(r["error"], "query")
        if not r["overflow"]:
            n = r["count"]
            return (fid[:n], tid[:n], offs) if offs is not None else (fid[:n], tid[:n])
        cap = query_capacity(r["required"], mode, **chunk)
    raise _lib.CrtError(_lib.CRT_ERR_OUTPUT_OVERFLOW, "query")


def query_stream(d_rt: RTree, d_rbox: BBox, d_qbox: BBox, consume, capacity: int = 1 << 30,
                 batch: int = 1 << 16, mode: int = _lib.CRT_QUERY_PERSISTENT, stream=None,
                 **opts) -> dict:
    """Queries a window set whose pairs need not fit in memory at once: the
    windows go through crt_query_into_f32 in consecutive batches against one
    fixed output buffer of `capacity` pairs.  A batch that overflows is run
    again on fewer windows (the result block reports the exact pair count it
    needed, so the retry is sized from it); after a batch that used less than
    half the buffer the next batch grows.  For each completed batch
    `consume(fid, tid, first)` receives device views of its pairs (tid
    relative to window `first`), before the buffer is reused.  A single
    window with more than `capacity` pairs is CRT_ERR_OUTPUT_OVERFLOW.
    Returns {"pairs", "batches", "retries"}."""
    nq = d_qbox.sz
    cap = int(capacity)
    # pairs a batch may need and still fit: the persistent form reserves
    # output in per-warp chunks, which may leave one partly used chunk each
    usable = cap - query_capacity(0, mode, **({"chunk": opts["chunk"]} if "chunk" in opts else {}))
    if usable <= 0:
        raise _lib.CrtError(_lib.CRT_ERR_INVALID_ARG,
                            f"query_stream: capacity {cap} is below the form's slack")
    fid = torch.empty(cap, dtype=torch.int32, device="cuda")
    tid = torch.empty(cap, dtype=torch.int32, device="cuda")
    res = new_result_block()
    h_res = torch.empty(64, dtype=torch.uint8, pin_memory=True)
    st = {"pairs": 0, "batches": 0, "retries": 0}
    a, size = 0, max(1, int(batch))
    while a < nq:
        b = min(nq, a + size)
        sub = BBox(d_qbox.xmin[a:b], d_qbox.ymin[a:b], d_qbox.xmax[a:b], d_qbox.ymax[a:b],
                   d_qbox.id[a:b])
        query_into(d_rt, d_rbox, sub, fid, tid, res, None, mode, stream, **opts)
        h_res.copy_(res)
        r = read_result(h_res)
        if r["error"]:
            raise _lib.CrtError(r["error"], "query_stream")
        if r["overflow"]:
            st["retries"] += 1
            if b - a == 1:
                raise _lib.CrtError(_lib.CRT_ERR_OUTPUT_OVERFLOW,
                                    f"query_stream: window {a} alone has {r['required']} pairs")
            size = max(1, min(b - a - 1, int((b - a) * 0.85 * usable / max(r["required"], 1))))
            continue
        n = r["count"]
        consume(fid[:n], tid[:n], a)
        st["pairs"] += n
        st["batches"] += 1
        a = b
        if 2 * n < usable:
            size = min(max(int(batch), 1) * 64, 2 * size)
    return st


def query_stats(d_rt: RTree, d_rbox: BBox, d_qbox: BBox, per_window: bool = False,
                stream=None):
    """Hit count and leaf boxes tested (by the reference's algorithm, and with
    the containment shortcut), in total (and per window)."""
    tot = (ctypes.c_int64 * 4)()
    hits = tested = None
    if per_window and d_qbox.sz:
        hits = torch.empty(d_qbox.sz, dtype=torch.int64, device="cuda")
        tested = torch.empty(d_qbox.sz, dtype=torch.int64, device="cuda")
    rb, qb = d_rbox.c(), d_qbox.c()
    check(load().crt_query_stats_f32(ctypes.byref(d_rt.s), ctypes.byref(rb), ctypes.byref(qb),
                                     hits.data_ptr() if hits is not None else None,
                                     tested.data_ptr() if tested is not None else None, tot,
                                     _stream_handle(stream)), "query_stats")
    out = {"hits": int(tot[0]), "tested": int(tot[1]), "tested_contain": int(tot[2]),
           "range_hits": int(tot[3])}
    if per_window:
        out["per_window_hits"] = hits
        out["per_window_tested"] = tested
    return out


class Plan:
    """A persistent query recorded once as a CUDA graph and replayed."""

    def __init__(self, d_rt: RTree, d_rbox: BBox, d_qbox: BBox, fid, tid, result,
                 stream=None, **opts):
        o = _lib.default_opts(**opts)
        self._keep = (d_rt, d_rbox, d_qbox, fid, tid, result)
        rb, qb = d_rbox.c(), d_qbox.c()
        h = ctypes.c_void_p()
        check(load().crt_plan_create(ctypes.byref(d_rt.s), ctypes.byref(rb), ctypes.byref(qb),
                                     d_qbox.sz, fid.data_ptr(), tid.data_ptr(), int(fid.numel()),
                                     result.data_ptr(), ctypes.byref(o), _stream_handle(stream),
                                     ctypes.byref(h)), "plan_create")
        self.h = h

    def launch(self, stream=None) -> None:
        check(load().crt_plan_launch(self.h, _stream_handle(stream)), "plan_launch")

    def set_nq(self, nq: int, stream=None) -> None:
        check(load().crt_plan_set_nq(self.h, nq, _stream_handle(stream)), "plan_set_nq")

    def destroy(self) -> None:
        if self.h:
            load().crt_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def read_mbr_csv(path: str, n: int = -1, r: float = 0.0, stream=None) -> BBox:
    """readMBR (src/utility.cpp:5-40) followed by box_h2d
    (src/utility.cuh:42-66), on the GPU: the records "x1,y1,x2,y2,id,pid,nume"
    of the file become the device box set [min(x1,x2) - r, max(x1,x2) + r] x
    [min(y1,y2) - r, max(y1,y2) + r] with the fifth field as id.  n = -1 reads
    every record; otherwise exactly n records must be present.  A malformed
    record or a short file raises CrtError (the reference exits or throws)."""
    return _read_mbr("crt_read_mbr_csv_device", path, n, r, stream)


def read_mbr_bin(path: str, n: int = -1, r: float = 0.0, stream=None) -> BBox:
    """The binary form of read_mbr_csv: 28-byte little-endian records of
    float32 x1, y1, x2, y2 and int32 id, pid, nume (datasets.mbr_bin_bytes
    writes them), the same boxes and ids as the text form of those values."""
    return _read_mbr("crt_read_mbr_bin_device", path, n, r, stream)


def _read_mbr(fn: str, path, n: int, r: float, stream) -> BBox:
    L = load()
    box = _lib.crt_bbox_f32()
    got = ctypes.c_int64(0)
    check(getattr(L, fn)(str(path).encode(), n, r, ctypes.byref(box), ctypes.byref(got),
                         _stream_handle(stream)), fn)
    try:
        out = BBox.empty(int(box.sz))
        if box.sz:
            for dst, src in ((out.xmin, box.xmin), (out.ymin, box.ymin), (out.xmax, box.xmax),
                             (out.ymax, box.ymax), (out.id, box.id)):
                _copy_ptr(dst.data_ptr(), src, 4 * int(box.sz))
    finally:
        L.crt_bbox_free(ctypes.byref(box))
    return out


def kernel_launches() -> int:
    return int(load().crt_kernel_launches())
