"""Autotuner for the persistent window query.

Picks, for one box set and a sample of its windows: the fanout of the tree
(every fanout gives the same pair set; it trades tree depth against wasted
leaf tests), the warps per CTA of the persistent traversal, whether the top
levels are staged in shared memory, and the output chunk a warp reserves.
Each candidate tree is built once (out of place, so the input is untouched);
each configuration is timed with CUDA events over a few repetitions and the
fastest median wins.  Results are cached in a JSON file keyed by the device
name and the workload's size class, so a process that has tuned once starts
with the winner.
"""
from __future__ import annotations

import json
import math
import os
import statistics

from . import _lib
from .rtree import BBox, build_into, new_result_block, query_capacity, query_into, query_stats

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "crtree_autotune.json")


def _key(device: str, nbox: int, nq: int) -> str:
    # size classes: powers of two of the box and window counts
    return f"{device}|boxes~2^{round(math.log2(max(nbox, 1)))}|windows~2^{round(math.log2(max(nq, 1)))}"


def autotune(d_boxes: BBox, d_windows: BBox, fanouts=(8, 16, 32), warps=(8, 16, 32),
             stage=(1, 0), chunks=(4096,), reps: int = 3, cache_path: str | None = DEFAULT_CACHE,
             use_cache: bool = True) -> dict:
    """Returns {"fanout", "warps_per_cta", "stage_levels", "chunk", "ms", "table"}."""
    import torch

    device = torch.cuda.get_device_name()
    key = _key(device, d_boxes.sz, d_windows.sz)
    if use_cache and cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cached = json.load(f).get(key)
        if cached:
            return dict(cached, cached=True)

    table = []
    best = None
    for f in fanouts:
        sorted_boxes, rt = build_into(d_boxes, f)
        pairs = query_stats(rt, sorted_boxes, d_windows)["hits"]
        cap = query_capacity(pairs)
        fid = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        tid = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        res = new_result_block()
        for w in warps:
            for st in stage:
                for ch in chunks:
                    opts = {"warps_per_cta": w, "stage_levels": st, "chunk": ch}
                    times = []
                    for r in range(reps + 1):
                        e0 = torch.cuda.Event(enable_timing=True)
                        e1 = torch.cuda.Event(enable_timing=True)
                        e0.record()
                        query_into(rt, sorted_boxes, d_windows, fid[:cap], tid[:cap], res, **opts)
                        e1.record()
                        e1.synchronize()
                        if r:  # the first run warms the pool and caches
                            times.append(e0.elapsed_time(e1))
                    ms = statistics.median(times)
                    row = {"fanout": f, **opts, "ms": ms}
                    table.append(row)
                    if best is None or ms < best["ms"]:
                        best = dict(row)
        del fid, tid, sorted_boxes, rt
        torch.cuda.empty_cache()
    best["table"] = table
    best["key"] = key
    if cache_path:
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        data = {}
        if os.path.exists(cache_path):
            with open(cache_path) as fh:
                try:
                    data = json.load(fh)
                except json.JSONDecodeError:
                    data = {}
        data[key] = {k: v for k, v in best.items() if k != "table"}
        with open(cache_path, "w") as fh:
            json.dump(data, fh, indent=1)
    return best


def query_opts(best: dict) -> dict:
    """The winner as keyword options for query/query_into/Plan."""
    return {"warps_per_cta": best["warps_per_cta"], "stage_levels": best["stage_levels"],
            "chunk": best["chunk"]}


__all__ = ["autotune", "query_opts", "DEFAULT_CACHE", "_lib"]
