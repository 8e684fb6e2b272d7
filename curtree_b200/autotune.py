"""Autotuner for the persistent window query.

Picks, for one box set and a sample of its windows: the fanout of the tree
(every fanout gives the same pair set; it trades tree depth against wasted
leaf tests), the warps per CTA of the persistent traversal, how many whole
tree levels are staged in shared memory, how many warps share one window,
and the output chunk a warp reserves (the frontier itself needs no
capacity: each warp's stack is sized exactly from the tree's depth).
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


def _time(fn, reps):
    import torch
    times = []
    for r in range(reps + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        if r:  # the first run warms the pool and caches
            times.append(e0.elapsed_time(e1))
    return statistics.median(times)


def autotune(d_boxes: BBox, d_windows: BBox, fanouts=(8, 16, 32), warps=(8, 16, 32),
             stage=(0, 1, 2, 3, 4), window_warps=(1, 2, 4), chunks=(1024, 4096, 16384),
             reps: int = 3, cache_path: str | None = DEFAULT_CACHE, use_cache: bool = True) -> dict:
    """Returns {"fanout", "warps_per_cta", "stage_levels", "warps_per_window",
    "chunk", "ms", "table"}.  The search goes one dimension at a time, each
    from the best so far: fanout x warps per CTA (every pair), then the
    staging depth in whole levels, then the warps sharing a window, then the
    output chunk; the table lists every configuration timed."""
    import torch

    device = torch.cuda.get_device_name()
    key = _key(device, d_boxes.sz, d_windows.sz)
    if use_cache and cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cached = json.load(f).get(key)
        if cached:
            return dict(cached, cached=True)

    table = []
    trees = {}

    def run(f, opts):
        if f not in trees:
            for old in list(trees):  # one candidate tree on the device at a time
                del trees[old]
            torch.cuda.empty_cache()
            sorted_boxes, rt = build_into(d_boxes, f)
            pairs = query_stats(rt, sorted_boxes, d_windows)["hits"]
            cap = max(query_capacity(pairs), query_capacity(pairs) + 64 * 16384 * 148)
            trees[f] = (sorted_boxes, rt, torch.empty(max(cap, 1), dtype=torch.int32, device="cuda"),
                        torch.empty(max(cap, 1), dtype=torch.int32, device="cuda"),
                        new_result_block())
        sb, rt, fid, tid, res = trees[f]
        ms = _time(lambda: query_into(rt, sb, d_windows, fid, tid, res, **opts), reps)
        row = {"fanout": f, **opts, "ms": ms}
        table.append(row)
        return row

    base = {"warps_per_cta": warps[0], "stage_levels": 2, "warps_per_window": 1, "chunk": 4096}
    best = None
    for f in fanouts:
        for w in warps:
            row = run(f, dict(base, warps_per_cta=w))
            if best is None or row["ms"] < best["ms"]:
                best = dict(row)
    for dim, values in (("stage_levels", stage), ("warps_per_window", window_warps),
                        ("chunk", chunks)):
        cur = {k: best[k] for k in base}
        for v in values:
            if v == cur[dim]:
                continue
            row = run(best["fanout"], dict(cur, **{dim: v}))
            if row["ms"] < best["ms"]:
                best = dict(row)
    trees.clear()
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
            "warps_per_window": best.get("warps_per_window", 1), "chunk": best["chunk"]}


__all__ = ["autotune", "query_opts", "DEFAULT_CACHE", "_lib"]
