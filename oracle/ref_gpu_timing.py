"""Times the reference's own GPU path beside this library's drop-in calls on
the same B200 and the same inputs (measurement infrastructure only).

Cases (seeded synthetic inputs, coordinates scaled by 2^15):
  small    1M uniform boxes (side U[0,1e-3]), 10k windows (side U[0,1e-2]),
           fanout 10: build_rtree + bfs_frontier, build_rtree + bfs_thrust;
  build    100M clustered boxes (1000 Gaussians + 10% uniform, log-normal
           sides, 1% duplicates, 1% points), fanout 10: build_rtree;
  batched  10M uniform boxes, 1M mixed windows (side log-U[1e-5,1e-1], half
           on box centres), fanout 10: bfs_frontier.
The reference runners (oracle/_ref, built by `make -C oracle ref`) time
build_rtree and the query with CUDA events on device-resident inputs, query
allocations included; this library is timed the same way through
crt_build_f32 and crt_query_f32 (in-place build, allocating query), and for
the batched case, whose pairs pass 2^31, through the persistent
crt_query_into_f32.  Each case also checks that both produce the same node
arrays and pair sets.

    python oracle/ref_gpu_timing.py [--cases small,build,batched] [--out FILE]

Prints one JSON object per case.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from curtree_b200 import datasets as D  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref_gpu as R  # noqa: E402


def ours(boxes, windows, fanout, reps, dropin=True):
    """Median build and query ms of this library, and its outputs.  dropin:
    crt_query_f32 (allocating, int32 pair count); otherwise the persistent
    crt_query_into_f32 into a buffer sized once (int64 pair count)."""
    import torch

    import curtree_b200 as C
    bms, qms = [], []
    tree = ids = pairs = None
    fid = tid = res = None
    count = None
    for r in range(reps + 1):
        d = C.BBox.from_host(boxes)
        rt = C.RTree(fanout)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        C.build_rtree(d, rt)
        e1.record()
        e1.synchronize()
        if r:
            bms.append(e0.elapsed_time(e1))
        if windows is not None:
            dq = C.BBox.from_host(windows)
            if not dropin and fid is None:
                cap = C.query_capacity(C.query_stats(rt, d, dq)["hits"])
                fid = torch.empty(cap, dtype=torch.int32, device="cuda")
                tid = torch.empty(cap, dtype=torch.int32, device="cuda")
                res = C.new_result_block()
            torch.cuda.synchronize()
            e0.record()
            if dropin:
                dp = C.bfs_frontier(rt, d, dq)
            else:
                C.query_into(rt, d, dq, fid, tid, res)
            e1.record()
            e1.synchronize()
            if r:
                qms.append(e0.elapsed_time(e1))
            if dropin:
                count = dp.sz
                if r == reps:
                    pairs = dp.to_host()
                dp.free()
            else:
                rr = C.read_result(res)
                assert rr["overflow"] == 0 and rr["error"] == 0, rr
                count = rr["count"]
        if r == reps:
            tree = rt.to_host()
            ids = d.id.cpu().numpy()
        rt.free()
        del d
        torch.cuda.empty_cache()
    med = lambda xs: statistics.median(xs) if xs else None
    return {"build_ms": med(bms), "query_ms": med(qms), "pairs": count,
            "query_call": "crt_query_f32" if dropin else "crt_query_into_f32 (persistent)"}, \
        tree, ids, pairs


def same_tree(ref_tree, ref_ids, tree, ids) -> bool:
    keys = ("xmin", "ymin", "xmax", "ymax", "pos", "len")
    return all(np.array_equal(np.asarray(ref_tree[k]).view(np.int32),
                              np.asarray(getattr(tree, k)).view(np.int32))
               for k in keys) and np.array_equal(ref_ids, ids)


def case(name, boxes, windows, fanout, runners, reps, tmp, dropin=True):
    bfile = os.path.join(tmp, name + "_boxes.crtb")
    boxes.write_crtb(bfile)
    qfile = None
    if windows is not None:
        qfile = os.path.join(tmp, name + "_windows.crtb")
        windows.write_crtb(qfile)
    mine, tree, ids, pairs = ours(boxes, windows, fanout, reps, dropin)
    out = {"case": name, "boxes": boxes.n, "windows": None if windows is None else windows.n,
           "fanout": fanout, "ours": mine, "reference": {}}
    cp = O.canonical_pairs(*pairs) if pairs is not None else None
    for runner in runners:
        mode = "query" if windows is not None else "build"
        try:
            t, rids, rp, info = R.run(runner, mode, bfile, qfile, fanout,
                                      os.path.join(tmp, name + "_" + runner), reps=reps)
        except R.RefRunFailed as e:
            tail = [ln for ln in (e.stdout + e.stderr).splitlines() if ln.strip()][-3:]
            out["reference"][runner] = {"failed": f"exit {e.rc}", "output_tail": tail}
            continue
        rec = {"build_ms": statistics.median(info["build_ms"]),
               "query_ms": statistics.median(info["query_ms"]) if info["query_ms"] else None,
               "tree_identical": same_tree(t, rids, tree, ids)}
        if rp is not None and cp is not None:
            rec["pairs"] = int(len(rp[0]))
            rc = O.canonical_pairs(*rp)
            rec["pairs_identical"] = bool(np.array_equal(rc[0], cp[0]) and np.array_equal(rc[1], cp[1]))
        out["reference"][runner] = rec
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default="small,build,batched")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    if not R.available("ref_frontier"):
        sys.exit("oracle/_ref/ref_frontier is missing: run `make -C oracle ref` where the "
                 "reference sources are present")
    import torch
    results = []
    with tempfile.TemporaryDirectory() as tmp:
        for name in args.cases.split(","):
            if name == "small":
                b = D.uniform_boxes(1_000_000, seed=1)
                q = D.uniform_windows(10_000, seed=101)
                r = case(name, b, q, 10, ["ref_frontier", "ref_thrust"], args.reps, tmp)
            elif name == "build":
                b = D.clustered_boxes(100_000_000, seed=2)
                r = case(name, b, None, 10, ["ref_frontier"], args.reps, tmp)
            elif name == "batched":
                b = D.uniform_boxes(10_000_000, seed=3)
                q = D.mixed_windows(1_000_000, b, seed=103)
                r = case(name, b, q, 10, ["ref_frontier"], 1, tmp, dropin=False)
            else:
                raise SystemExit(f"unknown case {name}")
            r["device"] = torch.cuda.get_device_name()
            print(json.dumps(r), flush=True)
            results.append(r)
            for f in os.listdir(tmp):
                p = os.path.join(tmp, f)
                shutil.rmtree(p) if os.path.isdir(p) else os.remove(p)
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(results, fh, indent=1)


if __name__ == "__main__":
    main()
