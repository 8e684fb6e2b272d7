"""Python view of the serving loop (crt_server_* in include/crtree.h):
continuous batching of window-query requests against device-resident trees,
admission by HBM footprint, overflow-and-retry, p50/p99 latency."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, load
from .rtree import BBox, RTree, _d2h


class Server:
    def __init__(self, arena_bytes: int = 8 << 30, max_requests: int = 4096,
                 max_trees: int = 16, pairs_per_window: float = 64.0,
                 output_slack: float = 1.5, idle_ms: int = 20, device_wait_us: int = 2_000_000):
        o = _lib.crt_server_opts()
        load().crt_server_opts_default(ctypes.byref(o))
        o.arena_bytes = arena_bytes
        o.max_requests = max_requests
        o.max_trees = max_trees
        o.pairs_per_window = pairs_per_window
        o.output_slack = output_slack
        o.idle_ms = idle_ms
        o.device_wait_us = device_wait_us
        h = ctypes.c_void_p()
        check(load().crt_server_create(ctypes.byref(o), ctypes.byref(h)), "server_create")
        self.h = h
        self._trees = []
        self._windows = {}

    def add_tree(self, rt: RTree, rbox: BBox) -> int:
        tid = ctypes.c_int(-1)
        rb = rbox.c()
        check(load().crt_server_add_tree(self.h, ctypes.byref(rt.s), ctypes.byref(rb),
                                         ctypes.byref(tid)), "server_add_tree")
        self._trees.append((rt, rbox))
        return int(tid.value)

    def submit(self, tree_id: int, windows) -> int | None:
        """Admit a window batch (HostBoxes or device BBox); None when the server
        is busy (no slot or arena space now)."""
        if isinstance(windows, BBox):
            ptrs = [windows.xmin.data_ptr(), windows.ymin.data_ptr(), windows.xmax.data_ptr(),
                    windows.ymax.data_ptr()]
            keep = None
        else:
            keep = [np.ascontiguousarray(a, dtype=np.float32)
                    for a in (windows.xmin, windows.ymin, windows.xmax, windows.ymax)]
            ptrs = [a.ctypes.data for a in keep]
        rid = ctypes.c_int64(-1)
        st = load().crt_server_submit(self.h, tree_id, *ptrs, windows.n if hasattr(windows, "n")
                                      else windows.sz, ctypes.byref(rid))
        if st == _lib.CRT_ERR_BUSY:
            return None
        check(st, "server_submit")
        return int(rid.value)

    def poll(self, max_out: int = 256, wait_ms: int = 0) -> list[dict]:
        buf = (_lib.crt_server_completion * max_out)()
        n = ctypes.c_int(0)
        check(load().crt_server_poll(self.h, buf, max_out, ctypes.byref(n), wait_ms), "server_poll")
        out = []
        for i in range(n.value):
            c = buf[i]
            out.append({"request_id": int(c.request_id), "tree_id": int(c.tree_id),
                        "status": int(c.status), "nq": int(c.nq), "count": int(c.count),
                        "d_fid": int(c.d_fid or 0), "d_tid": int(c.d_tid or 0),
                        "submit_time_s": float(c.submit_time_s),
                        "complete_time_s": float(c.complete_time_s), "retries": int(c.retries)})
        return out

    @staticmethod
    def pairs(completion: dict) -> tuple[np.ndarray, np.ndarray]:
        n = completion["count"]
        return _d2h(completion["d_fid"], n, np.int32), _d2h(completion["d_tid"], n, np.int32)

    def release(self, request_id: int) -> None:
        check(load().crt_server_release(self.h, request_id), "server_release")

    def stats(self) -> dict:
        v = [ctypes.c_int64(0) for _ in range(4)]
        st = load().crt_server_stats(self.h, *[ctypes.byref(x) for x in v])
        return {"submitted": v[0].value, "completed": v[1].value, "retried": v[2].value,
                "arena_used": v[3].value, "device_status": int(st)}

    def close(self) -> int:
        st = 0
        if self.h:
            st = load().crt_server_destroy(self.h)
            self.h = None
        return st

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
