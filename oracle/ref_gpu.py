"""Runs the reference's own GPU code path (test and measurement
infrastructure only).

`make -C oracle ref` compiles the reference's `build_rtree` with
`bfs_frontier` (oracle/_ref/ref_frontier) and with `bfs_thrust`
(oracle/_ref/ref_thrust) from its sources (src/rtree_bulkload_thrust.cuh,
src/rtree_bfs_frontier.cuh, src/rtree_bfs_thrust.cuh).  Each runner reads
CRTB box files, times the reference calls with CUDA events and writes the
node arrays, the permuted box ids and the hit pairs.  Nothing here is part of
the library's product path.
"""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref")


class RefRunFailed(RuntimeError):
    """The runner exited non-zero (the reference exits on its own limits,
    such as a full frontier queue)."""

    def __init__(self, cmd, rc, stdout, stderr):
        super().__init__(f"{' '.join(cmd)} -> exit {rc}\n{stdout[-1500:]}\n{stderr[-1500:]}")
        self.rc = rc
        self.stdout = stdout
        self.stderr = stderr


def available(runner: str = "ref_frontier") -> bool:
    return os.access(os.path.join(REF_BIN, runner), os.X_OK)


def run(runner: str, mode: str, bfile: str, qfile: str | None, fanout: int, outdir: str,
        reps: int = 1, timeout: float = 900, want_pairs: bool = True):
    """Runs `runner` ("ref_frontier" or "ref_thrust") in `mode` ("build" or
    "query").  Returns (tree dict of node arrays, sorted box ids, pairs
    (fid, tid) or None, info dict with build_ms / query_ms per repetition)."""
    os.makedirs(outdir, exist_ok=True)
    cmd = [os.path.join(REF_BIN, runner), mode, bfile, qfile or "-", str(fanout), outdir, str(reps)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RefRunFailed(cmd, p.returncode, p.stdout, p.stderr)
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("REFJSON ")][-1]
    info = json.loads(line[len("REFJSON "):])
    tree = np.fromfile(os.path.join(outdir, "tree.bin"), np.uint8)
    rsz = int(tree[:8].view(np.int64)[0])
    body = tree[16:]

    def arr(k, dt):
        return body[k * 4 * rsz:(k + 1) * 4 * rsz].view(dt)

    t = {"xmin": arr(0, np.float32), "ymin": arr(1, np.float32), "xmax": arr(2, np.float32),
         "ymax": arr(3, np.float32), "pos": arr(4, np.int32), "len": arr(5, np.int32)}
    ids = np.fromfile(os.path.join(outdir, "sorted_ids.bin"), np.int32)
    pairs = None
    if mode == "query" and want_pairs:
        raw = np.fromfile(os.path.join(outdir, "pairs.bin"), np.uint8)
        m = int(raw[:8].view(np.int64)[0])
        pairs = (raw[8:8 + 4 * m].view(np.int32), raw[8 + 4 * m:8 + 8 * m].view(np.int32))
    return t, ids, pairs, info
