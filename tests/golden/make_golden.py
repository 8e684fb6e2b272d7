"""Generate the golden fixtures from the reference's own GPU code path.

Runs oracle/_ref/ref_frontier and oracle/_ref/ref_thrust (build_rtree +
bfs_frontier / bfs_thrust compiled from the reference sources by
`make -C oracle ref`) on a B200 over small seeded inputs and stores, per case:
the inputs, the fanout, the node arrays, the sorted box ids and the canonical
(window, box id) hit pairs of each query path.

    python tests/golden/make_golden.py <outdir>

The fixtures in tests/golden/*.npz were made by this script; the tests read
them without the reference or a GPU.  Cases the reference cannot run are not
attempted: one box (its rt_d_alloc asserts on an empty tree), queries whose
32-window blocks would expand past its 1024-slot queue (it exits), and Thrust
queries where no window reaches a leaf-parent (its final filter then indexes
the box arrays with negative slots).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from curtree_b200 import datasets as D  # noqa: E402
from curtree_b200.datasets import HostBoxes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref_gpu as R  # noqa: E402

def boxes_from(xmin, ymin, xmax, ymax) -> HostBoxes:
    f = lambda a: np.asarray(a, np.float32)
    n = len(xmin)
    return HostBoxes(f(xmin), f(ymin), f(xmax), f(ymax), np.arange(n, dtype=np.int32))


def cases():
    out = []
    b = D.uniform_boxes(20000, seed=1)
    q = D.uniform_windows(500, seed=101)
    # windows that coincide with boxes: touching edges on every side
    q = HostBoxes.concat([q, b.take(np.arange(0, 20000, 400))])
    q.id = np.arange(q.n, dtype=np.int32)
    out.append(("uniform_20k", b, q, 10, True))
    b2 = D.uniform_boxes(10007, seed=11)
    q2 = D.uniform_windows(200, seed=111)
    for f in (2, 3, 8, 16, 32):
        out.append((f"fanout_{f}", b2, q2, f, True))
    for n, f in ((2, 2), (7, 10), (10, 10), (11, 10), (101, 10)):
        bb = D.uniform_boxes(n, seed=20 + n)
        qq = D.uniform_windows(64, seed=120 + n, max_side=0.5)
        out.append((f"small_n{n}_f{f}", bb, qq, f, True))
    # centres at or above 2^15: bit 31 of the key set -> negative signed keys
    rng = np.random.default_rng(7)
    cx = rng.uniform(0, 65536, 6000)
    cy = rng.uniform(0, 65536, 6000)
    w = rng.uniform(0, 40, 6000)
    out.append(("signed_keys", boxes_from(cx - w, cy - w, cx + w, cy + w),
                boxes_from(*(lambda c, d, s: (c - s, d - s, c + s, d + s))(
                    rng.uniform(0, 65536, 100), rng.uniform(0, 65536, 100),
                    rng.uniform(0, 300, 100))), 10, True))
    # raw [0,1) data: every key 0, identity order, whole-domain nodes
    out.append(("raw_unit", D.uniform_boxes(5000, seed=3, scale=False), None, 10, False))
    # duplicates, zero-area boxes, negative and huge coordinates (key saturation)
    rng = np.random.default_rng(9)
    n = 4000
    cx = rng.uniform(-2000, 70000, n)
    cy = rng.uniform(-2000, 70000, n)
    w = rng.uniform(0, 50, n)
    w[::7] = 0.0
    xs = [cx - w, cy - w, cx + w, cy + w]
    for a in xs:
        a[100:200] = a[50]
    out.append(("specials", boxes_from(*xs),
                boxes_from(*(lambda c, d, s: (c - s, d - s, c + s, d + s))(
                    rng.uniform(-2000, 70000, 80), rng.uniform(-2000, 70000, 80),
                    rng.uniform(0, 400, 80))), 10, True))
    # centres far outside the 16-bit range, up to beyond 2^32, and far negative
    rng = np.random.default_rng(10)
    n = 3000
    mag = np.exp(rng.uniform(np.log(1.0), np.log(1e11), n)) * np.where(rng.random(n) < 0.2, -1, 1)
    cy = rng.uniform(0, 70000, n)
    w = rng.uniform(0, 10, n)
    out.append(("huge_coords", boxes_from(mag - w, cy - w, mag + w, cy + w), None, 10, False))
    # NaN coordinates and signed zeros: build only
    xs = [a.copy() for a in xs]
    xs[0][300:310] = np.nan
    xs[3][400:405] = np.nan
    xs[0][500:520] = -0.0
    xs[2][500:520] = 0.0
    xs[1][520:540] = 0.0
    xs[3][520:540] = -0.0
    out.append(("nan_zero", boxes_from(*xs), None, 10, False))
    return out


def run(runner, mode, bfile, qfile, fanout, outdir):
    t, ids, pairs, info = R.run(runner, mode, bfile, qfile, fanout, outdir, reps=1, timeout=600)
    if pairs is not None:
        pairs = O.canonical_pairs(*pairs)
    return t, ids, pairs, info


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    tmp = tempfile.mkdtemp()
    summary = {}
    for name, b, q, f, do_query in cases():
        bfile = os.path.join(tmp, name + "_boxes.crtb")
        b.write_crtb(bfile)
        qfile = None
        if q is not None:
            qfile = os.path.join(tmp, name + "_windows.crtb")
            q.write_crtb(qfile)
        rec = {"fanout": np.int32(f)}
        for k in ("xmin", "ymin", "xmax", "ymax", "id"):
            rec["box_" + k] = getattr(b, k)
            if q is not None:
                rec["win_" + k] = getattr(q, k)
        # oracle view, to decide which reference query paths are safe to run
        sb, tr = O.build(b, f)
        run_frontier = run_thrust = False
        if do_query and q is not None:
            st = O.tree_query_stats(tr, sb, q)
            run_frontier = st.total > 0
            run_thrust = st.tested.sum() > 0
        try:
            t, ids, pairs, info = run("ref_frontier", "query" if run_frontier else "build",
                                      bfile, qfile, f, os.path.join(tmp, name + "_f"))
        except RuntimeError as e:
            if not run_frontier:
                raise
            # the frontier queue overflowed (the reference exits): keep the build
            print(name, "frontier query failed:", str(e).splitlines()[0], flush=True)
            t, ids, pairs, info = run("ref_frontier", "build", bfile, None, f,
                                      os.path.join(tmp, name + "_f"))
        for k, v in t.items():
            rec["node_" + k] = v
        rec["sorted_id"] = ids
        if pairs is not None:
            rec["frontier_fid"], rec["frontier_tid"] = pairs
        if run_thrust:
            try:
                t2, ids2, pairs2, info2 = run("ref_thrust", "query", bfile, qfile, f,
                                              os.path.join(tmp, name + "_t"))
                assert all(np.array_equal(t[k].view(np.uint32), t2[k].view(np.uint32)) for k in t)
                rec["thrust_fid"], rec["thrust_tid"] = pairs2
            except RuntimeError as e:
                print(name, "thrust query failed:", str(e)[-300:], flush=True)
                run_thrust = False
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)
        summary[name] = {"n": b.n, "fanout": f, "r_sz": int(len(t["pos"])),
                         "frontier_pairs": None if pairs is None else int(len(pairs[0])),
                         "thrust": bool(run_thrust)}
        print(name, summary[name], flush=True)
    with open(os.path.join(outdir, "SUMMARY.json"), "w") as fh:
        json.dump(summary, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <outdir>")
    main(sys.argv[1])
