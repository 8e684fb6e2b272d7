"""Benchmark: batched window queries against a 10M-box tree on one B200 (or N
replicas), plus the 100M-box bulk load.

Headline (one JSON line on rank 0):
  metric  window queries/s of the persistent, graph-captured query form
          (10M uniform boxes, side U[0,1e-3]; 1M windows, side log-uniform in
          [1e-5, 1e-1], half centred on boxes, half uniform), every hit pair
          written to HBM.  A step = one pass over the 1M-window batch.
  plain   the same batch through the plain per-batch form (count pass, scan,
          write pass; one warp per window in input order).
  build   100M clustered boxes (1000 Gaussian clusters + 10% uniform,
          log-normal sides, 1% duplicates, 1% points): encode + radix sort +
          node build, boxes/s.
  e2e     the same query metric through the C ABI with host buffers: each step
          copies the windows from pinned host memory, queries, reads the pair
          count and copies every result back to pinned host memory (as CSR:
          ids + offsets, or as pairs; the faster is reported, with the other
          beside it).
  serving four resident trees (1M-50M boxes), 400 requests of 1-100k
          windows arriving as a Poisson stream at 1k, 3k and 10k requests/s:
          continuous batching against the plain form one request at a time,
          windows/s and p50/p99 latency.
  roofline  of the dominant kernel (the persistent traversal): algorithmic bytes
          16 B per window + 16 B per leaf box it tests + 12 B per hit, over
          its CUDA-event time, against the measured HBM copy bandwidth.
  cpu_baseline  the reference's own CPU brute force (nested_loop_query,
          compiled from its sources) on the host cores over a bounded sample.

`--impl reference` times that CPU path alone (rank 0) on the same metric.
All inputs are synthetic and seeded (no dataset is involved).  The box SoA
(200 MB), the windows and the output (tens of GB) are larger than L2, so no
flush is needed between steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

QUERY_BOXES = 10_000_000
QUERY_WINDOWS = 1_000_000
BUILD_BOXES = 100_000_000
FANOUT = 16


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--boxes", type=int, default=QUERY_BOXES)
    p.add_argument("--windows", type=int, default=QUERY_WINDOWS)
    p.add_argument("--build-boxes", type=int, default=BUILD_BOXES)
    p.add_argument("--fanout", type=int, default=FANOUT)
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--warps", type=int, default=0, help="warps per CTA of the persistent traversal")
    p.add_argument("--stage", type=int, default=1, help="stage the top tree levels in shared memory")
    p.add_argument("--sort-windows", type=int, default=1)
    p.add_argument("--autotune", type=int, default=1, help="pick fanout/warps/staging first (untimed)")
    p.add_argument("--autotune-windows", type=int, default=100_000)
    p.add_argument("--skip", default="",
                   help="comma list of legs to skip: build,e2e,plain,cpu,serve,adversarial")
    p.add_argument("--adv-boxes", type=int, default=50_000_000)
    p.add_argument("--adv-windows", type=int, default=2_000_000)
    p.add_argument("--adv-buffer-log2", type=int, default=32,
                   help="output buffer of the streamed adversarial leg: 2^k pairs")
    p.add_argument("--ingest-records", type=int, default=4_000_000,
                   help="records of the MBR text file the ingest leg reads")
    p.add_argument("--serve-trees", default="1000000,5000000,20000000,50000000")
    p.add_argument("--serve-requests", type=int, default=400)
    p.add_argument("--serve-rates", default="1000,3000,10000",
                   help="comma list of Poisson arrival rates (requests/s)")
    p.add_argument("--serve-max-batch", type=int, default=100_000)
    p.add_argument("--serve-arena-gb", type=int, default=64)
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        loaded = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference CPU path (bounded sample)
# ---------------------------------------------------------------------------
def cpu_reference_rate(boxes, windows, seconds: float, rng_seed: int = 7):
    """Windows/s of the reference's nested_loop_query over all host threads,
    on a sample of windows sized to about `seconds` of CPU work.  Falls back to
    the oracle's restatement when the reference build is absent."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    kind = "reference" if O.ref_cpu_available() else "port"
    rng = np.random.default_rng(rng_seed)

    def run(m):
        idx = np.sort(rng.choice(windows.n, size=min(m, windows.n), replace=False))
        q = windows.take(idx)
        qid = np.arange(q.n, dtype=np.int32)
        t0 = time.perf_counter()
        if kind == "reference":
            R = O.ref_cpu()
            a = [np.ascontiguousarray(x) for x in (q.xmin, q.ymin, q.xmax, q.ymax)]
            d = [np.ascontiguousarray(x) for x in (boxes.xmin, boxes.ymin, boxes.xmax, boxes.ymax)]
            pairs = R.ref_nested_loop_query_mt(*a, qid, q.n, *d, boxes.id, boxes.n, threads)
        else:
            c, _ = O.nested_loop_stats(q, boxes, nthreads=threads)
            pairs = int(c.sum())
        return q.n, time.perf_counter() - t0, int(pairs)

    n0, t0, _ = run(threads)
    m = int(max(threads, min(windows.n, n0 / max(t0, 1e-6) * seconds)))
    m = (m + threads - 1) // threads * threads
    n, t, pairs = run(m)
    return {"value": n / t, "unit": "windows/s", "cores": threads, "kind": kind,
            "sample": f"{n} of {windows.n} windows x {boxes.n} boxes, {t:.1f} s, {pairs} pairs"}


def cpu_rtree_rate(h_tree, h_sorted, windows, seconds: float, rng_seed: int = 9):
    """Windows/s of a CPU R-tree on all host threads: the same packed tree
    (the reference's layout, copied from the device) searched depth-first by
    the oracle's C restatement of the reference's tree query, counting hits
    and pair digests without writing pairs.  It stands in for the reference's
    Boost R-tree check (src/verify.hpp:35-104), whose Boost dependency is
    absent; a sample of windows sized to about `seconds` of CPU work."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(rng_seed)

    def run(m):
        idx = np.sort(rng.choice(windows.n, size=min(m, windows.n), replace=False))
        q = windows.take(idx)
        t0 = time.perf_counter()
        st = O.tree_query_stats(h_tree, h_sorted, q, nthreads=threads)
        return q.n, time.perf_counter() - t0, st.total

    n0, t0, _ = run(threads * 8)
    m = int(max(threads, min(windows.n, n0 / max(t0, 1e-6) * seconds)))
    m = (m + threads - 1) // threads * threads
    n, t, pairs = run(m)
    return {"value": n / t, "unit": "windows/s", "cores": threads, "kind": "port",
            "sample": f"{n} of {windows.n} windows x {h_sorted.n} boxes, {t:.1f} s, {pairs} pairs",
            "what": "depth-first search of the same packed tree on the host (oracle restatement "
                    "of the reference's query), hits counted, no pair writes"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def make_query_inputs(rank: int, nbox: int, nwin: int):
    from curtree_b200 import datasets as D
    boxes = D.uniform_boxes(nbox, seed=3)
    windows = D.mixed_windows(nwin, boxes, seed=103 + 1000 * rank)
    return boxes, windows


# A serving replay that has not finished by then is a fault, not a slow run.
SERVE_DEADLINE_S = 120.0


def traffic_for(kernel: str, units: float):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/traffic.json: bytes measured on a smaller launch and the units
    it processed), scaled to `units`; None when absent."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f).get(kernel)
    if not t:
        return None
    return t["dram_bytes"] * units / t["units"]


def reduce_max(x: float, dist, device="cuda") -> float:
    """Max of a per-rank value over all ranks (the step time the JSON line
    reports); the identity on one process."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed(fn, steps, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def profile_collect(name):
    import ctypes
    from curtree_b200 import _lib
    ms = ctypes.c_double(0)
    n = ctypes.c_int64(0)
    _lib.load().crt_profile_collect(name.encode() if name else None, ctypes.byref(ms), ctypes.byref(n))
    return ms.value, n.value


def run_ours(args, rank, world, dist):
    import ctypes

    import torch

    import curtree_b200 as C
    from curtree_b200 import _lib

    L = _lib.load()
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    skip = set(s for s in args.skip.split(",") if s)
    hbm_peak, peak_kind = peaks()
    out = {}

    # ---- inputs resident in HBM -------------------------------------------
    boxes, windows = make_query_inputs(rank, args.boxes, args.windows)
    d_in = C.BBox.from_host(boxes)
    tuned = None
    if args.autotune:
        # untimed: pick fanout / warps / staging on a sample of the windows
        from curtree_b200.autotune import autotune
        sample = windows.take(np.arange(0, windows.n, max(1, windows.n // args.autotune_windows)))
        tuned = autotune(d_in, C.BBox.from_host(sample), cache_path=None, reps=2)
        args.fanout = tuned["fanout"]
        args.warps = tuned["warps_per_cta"]
        args.stage = tuned["stage_levels"]
        torch.cuda.empty_cache()
    out["autotune"] = None if tuned is None else {
        "chosen": {k: tuned[k] for k in ("fanout", "warps_per_cta", "stage_levels", "chunk", "ms")},
        "sample_windows": int(sample.n),
        "table": [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in row.items()}
                  for row in tuned["table"]]}
    sorted_box, rt = C.build_into(d_in, args.fanout)
    del d_in
    d_win = C.BBox.from_host(windows)
    st = C.query_stats(rt, sorted_box, d_win)
    pairs, tested, tested_c = st["hits"], st["tested"], st["tested_contain"]
    cap = C.query_capacity(pairs)
    fid = torch.empty(cap, dtype=torch.int32, device="cuda")
    tid = torch.empty(cap, dtype=torch.int32, device="cuda")
    res = C.new_result_block()

    # ---- persistent form (graph plan) -------------------------------------
    L.crt_profile_enable(1)
    qopts = {"warps_per_cta": args.warps, "stage_levels": args.stage,
             "sort_windows": args.sort_windows}
    plan = C.Plan(rt, sorted_box, d_win, fid, tid, res, **qopts)
    for _ in range(args.warmup):
        plan.launch()
    torch.cuda.synchronize()
    r = C.read_result(res)
    assert r["overflow"] == 0 and r["count"] == pairs and r["error"] == 0, r
    profile_collect(None)
    launches0 = C.kernel_launches()
    if dist is not None:
        dist.barrier()
    with Clocks(dev) as clk:
        ms = timed(plan.launch, args.steps, stream)
    launches = C.kernel_launches() - launches0
    k_ms, k_n = profile_collect("traverse_persistent")
    profile_collect(None)
    r = C.read_result(res)
    assert r["overflow"] == 0 and r["count"] == pairs, r
    ms_max = reduce_max(ms, dist)
    step_ms = ms_max / args.steps
    kern_ms = k_ms / max(k_n, 1) if k_n else step_ms
    # per-unit figure of the window query: 16 B per window + 16 B per leaf box tested +
    # 12 B per hit (id read + pair write); the boxes tested are the ones this
    # kernel tests (containment emits contained subtrees without reading
    # their boxes); the reference algorithm's count and the strict I/O floor
    # are reported beside it
    alg_bytes = 16 * args.windows + 16 * tested_c + 12 * pairs
    ref_bytes = 16 * args.windows + 16 * tested + 12 * pairs
    rsz_q = C.tree_size(args.boxes, args.fanout)
    io_bytes = 16 * args.windows + 12 * pairs + 20 * args.boxes + 24 * rsz_q
    gbs = lambda b: b / (kern_ms / 1e3) / 1e9
    out["persistent"] = {"ms_per_step": step_ms, "windows_per_s": world * args.windows / (step_ms / 1e3),
                         "kernel_ms": kern_ms, "opts": qopts}
    out["roofline"] = {"bound": "hbm", "achieved": gbs(alg_bytes), "peak": hbm_peak, "unit": "GB/s",
                       "frac": gbs(alg_bytes) / hbm_peak, "traffic": traffic_for("persistent_kernel", pairs),
                       "peak_kind": peak_kind, "kernel": "persistent_kernel",
                       "algorithmic_bytes": alg_bytes,
                       "bytes_model": "16 B/window + 16 B/leaf box tested + 12 B/hit (boxes this kernel tests)",
                       "reference_algorithm": {"bytes": ref_bytes, "frac": gbs(ref_bytes) / hbm_peak,
                                               "note": "charges every leaf box the reference tests"},
                       "strict_io": {"bytes": io_bytes, "frac": gbs(io_bytes) / hbm_peak,
                                     "note": "windows + pair writes + id reads + one read of the tree"}}
    out["clocks"] = clk.summary()
    out["gpu_launches"] = launches
    out["workload_stats"] = {"pairs": pairs, "leaf_boxes_tested_reference": tested,
                             "leaf_boxes_tested": tested_c, "pairs_from_contained_ranges": st["range_hits"],
                             "pairs_per_window": pairs / args.windows}
    plan.destroy()

    # ---- plain form ---------------------------------------------------------
    if "plain" not in skip:
        offs = torch.empty(args.windows + 1, dtype=torch.int64, device="cuda")
        plain = lambda: C.query_into(rt, sorted_box, d_win, fid, tid, res, offs, C.CRT_QUERY_PLAIN)
        for _ in range(max(1, args.warmup)):
            plain()
        torch.cuda.synchronize()
        r = C.read_result(res)
        assert r["overflow"] == 0 and r["count"] == pairs, r
        profile_collect(None)
        pms = timed(plain, args.steps, stream)
        pk_ms, pk_n = profile_collect("traverse_plain")
        profile_collect(None)
        pms = reduce_max(pms, dist)
        out["plain"] = {"ms_per_step": pms / args.steps,
                        "windows_per_s": world * args.windows / (pms / args.steps / 1e3),
                        "kernel_ms": pk_ms / max(args.steps, 1)}
        del offs

    # ---- CPU R-tree on the same tree (rank 0 of a 1-GPU run) ------------------
    if "cpu" not in skip and rank == 0 and world == 1:
        try:
            out["cpu_rtree"] = cpu_rtree_rate(rt.to_host(), sorted_box.to_host(), windows,
                                              args.cpu_seconds)
        except Exception as e:  # a side figure: report it, keep the line
            out["cpu_rtree"] = {"error": f"{type(e).__name__}: {e}"}

    # ---- end to end through the C ABI with host buffers ----------------------
    if "e2e" not in skip:
        out["e2e"] = e2e_leg(args, C, L, rt, sorted_box, windows, pairs, fid, tid, res, stream,
                             dist, world)

    L.crt_profile_enable(0)
    del fid, tid
    torch.cuda.empty_cache()

    # ---- serving loop -----------------------------------------------------------
    if "serve" not in skip:
        out["serving"] = serving_leg(args, C, rank)
        torch.cuda.empty_cache()

    # ---- adversarial geometry ------------------------------------------------------
    if "adversarial" not in skip:
        out["adversarial"] = adversarial_leg(args, C, stream, dist, world, rank)
        torch.cuda.empty_cache()

    # ---- ingest: MBR text file -> device boxes ---------------------------------
    if "ingest" not in skip and rank == 0:
        out["ingest"] = ingest_leg(args, C, L, stream)
        torch.cuda.empty_cache()

    # ---- bulk load ------------------------------------------------------------
    if "build" not in skip:
        out["build"] = build_leg(args, C, L, hbm_peak, peak_kind, stream, dist, world)
    return out, boxes, windows


def e2e_leg(args, C, L, rt, sorted_box, windows, pairs, fid, tid, res, stream, dist, world):
    """End to end through the C ABI with host buffers, per step: the windows
    H2D from pinned host memory, the query, the result block D2H (the pair
    count), then every result D2H to pinned host memory.  Two result forms:
    CSR (plain form: box ids grouped by window + int64 offsets, 4 B per pair)
    and pairs (persistent form: box id + window index, 8 B per pair).  The
    faster is the headline e2e; both are reported."""
    import psutil
    import torch
    nwin = windows.n
    # every rank on this node pins its own result buffers: budget a share each
    local = max(1, int(os.environ.get("LOCAL_WORLD_SIZE", "1")))
    avail = psutil.virtual_memory().available / local
    if 8 * pairs * 1.5 > avail:
        return {"value": None, "unit": "windows/s",
                "skipped": f"host memory share {avail / 1e9:.0f} GB < 1.5 x {8 * pairs / 1e9:.0f} GB of pairs"}
    h_win = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
             for a in (windows.xmin, windows.ymin, windows.xmax, windows.ymax, windows.id)]
    h2d = sum(int(h.numel() * h.element_size()) for h in h_win)
    d_win = C.BBox.empty(nwin)
    dst = [d_win.xmin, d_win.ymin, d_win.xmax, d_win.ymax, d_win.id]
    h_res = torch.empty(64, dtype=torch.uint8, pin_memory=True)
    offs = torch.empty(nwin + 1, dtype=torch.int64, device="cuda")
    h_fid = torch.empty(pairs, dtype=torch.int32, pin_memory=True)

    def run(step, d2h_per_step, path):
        for _ in range(max(1, min(args.warmup, 2))):
            step()
        torch.cuda.synchronize()
        r = C.read_result(h_res)
        assert r["count"] == pairs and r["overflow"] == 0, r
        ms = reduce_max(timed(step, args.steps, stream), dist)
        return {"value": world * nwin / (ms / args.steps / 1e3), "unit": "windows/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h_per_step,
                "ms_per_step": ms / args.steps, "path": path}

    def h2d_windows():
        for d, h in zip(dst, h_win):
            d.copy_(h, non_blocking=True)

    def count():
        h_res.copy_(res, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return C.read_result(h_res)["count"]

    # CSR: box ids grouped by window and the offsets, two steps in flight:
    # step i's results cross PCIe while step i + 1 queries on the other
    # stream (each step still copies its windows in and all its results out)
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    sets = []
    for k in range(2):
        with torch.cuda.stream(streams[k]):
            w = C.BBox.empty(nwin)
            f = fid if k == 0 else torch.empty(pairs, dtype=torch.int32, device="cuda")
            sets.append({"win": w, "dst": [w.xmin, w.ymin, w.xmax, w.ymax, w.id], "fid": f,
                         "offs": torch.empty(nwin + 1, dtype=torch.int64, device="cuda"),
                         "res": C.new_result_block(),
                         "h_res": torch.empty(64, dtype=torch.uint8, pin_memory=True),
                         "h_fid": h_fid if k == 0 else torch.empty(pairs, dtype=torch.int32,
                                                                    pin_memory=True),
                         "h_offs": torch.empty(nwin + 1, dtype=torch.int64, pin_memory=True)})
    torch.cuda.synchronize()
    counter = [0]

    def step_csr():
        k = counter[0] % 2
        counter[0] += 1
        st, z = streams[k], sets[k]
        with torch.cuda.stream(st):
            for d, h in zip(z["dst"], h_win):
                d.copy_(h, non_blocking=True)
            C.query_into(rt, sorted_box, z["win"], z["fid"], None, z["res"], z["offs"],
                         C.CRT_QUERY_PLAIN, st)
            z["h_res"].copy_(z["res"], non_blocking=True)
            st.synchronize()  # the pair count sizes the copy out
            n = C.read_result(z["h_res"])["count"]
            z["h_offs"].copy_(z["offs"], non_blocking=True)
            z["h_fid"][:n].copy_(z["fid"][:n], non_blocking=True)

    def run_csr():
        for _ in range(max(1, min(args.warmup, 2))):
            step_csr()
        torch.cuda.synchronize()
        r = C.read_result(sets[0]["h_res"])
        assert r["count"] == pairs and r["overflow"] == 0, r
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step_csr()
        for st in streams:  # the last steps' copies out belong to the timed region
            stream.wait_stream(st)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = reduce_max(e0.elapsed_time(e1), dist)
        return {"value": world * nwin / (ms / args.steps / 1e3), "unit": "windows/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4 * pairs + 8 * (nwin + 1) + 64,
                "ms_per_step": ms / args.steps,
                "path": "crt_query_into_f32 (plain form, CSR: ids + offsets) via ctypes, "
                        "two steps in flight on two streams"}

    csr = run_csr()
    del sets, streams
    # pairs: box id and window index
    h_tid = torch.empty(pairs, dtype=torch.int32, pin_memory=True)

    def step_pairs():
        h2d_windows()
        C.query_into(rt, sorted_box, d_win, fid, tid, res)
        n = count()
        h_fid[:n].copy_(fid[:n], non_blocking=True)
        h_tid[:n].copy_(tid[:n], non_blocking=True)

    prs = run(step_pairs, 8 * pairs + 64, "crt_query_into_f32 (persistent form, pairs) via ctypes")
    best, other = (csr, prs) if csr["value"] >= prs["value"] else (prs, csr)
    return dict(best, alternative=other)


def serving_workload(args, rank):
    """Four device-resident trees (1M, 5M, 20M, 50M uniform boxes) and a
    request stream: tree uniform, batch size log-uniform in [1, 100k]
    windows, window side log-uniform in [1e-5, 1e-1]; exponential
    inter-arrival gaps of mean 1 (scaled by the rate)."""
    from curtree_b200 import datasets as D
    sizes = [int(x) for x in args.serve_trees.split(",")]
    trees = [D.uniform_boxes(n, seed=41 + i) for i, n in enumerate(sizes)]
    tree_idx, nq = D.serving_requests(args.serve_requests, len(trees), seed=104 + 1000 * rank,
                                      hi=args.serve_max_batch)
    rng = np.random.default_rng(204 + rank)
    gaps = np.cumsum(rng.exponential(1.0, args.serve_requests))
    reqs = []
    for i in range(args.serve_requests):
        w = D.mixed_windows(int(nq[i]), trees[tree_idx[i]], seed=10_000 + 7 * i + 1000 * rank)
        reqs.append((int(tree_idx[i]), w))
    return trees, reqs, gaps


def serve_run(srv, tids, reqs, arrivals):
    """Replays one arrival schedule through the server; returns latencies
    (arrival to completion), makespan, pairs and retries."""
    import time
    lat = np.zeros(len(reqs))
    pairs = retries = 0
    backlog, ids = [], {}
    nxt = done = 0
    t0 = time.monotonic()
    while done < len(reqs):
        now = time.monotonic() - t0
        if now > SERVE_DEADLINE_S:
            raise RuntimeError(f"serving run passed {SERVE_DEADLINE_S} s: {done} of {len(reqs)} done")
        while nxt < len(reqs) and arrivals[nxt] <= now:
            backlog.append(nxt)
            nxt += 1
        while backlog:
            i = backlog[0]
            rid = srv.submit(tids[reqs[i][0]], reqs[i][1])
            if rid is None:
                break
            ids[rid] = i
            backlog.pop(0)
        for c in srv.poll(max_out=256, wait_ms=0 if (backlog or nxt < len(reqs)) else 2):
            i = ids.pop(c["request_id"])
            if c["status"] != 0:
                raise RuntimeError(f"served request failed: {c}")
            lat[i] = c["complete_time_s"] - (t0 + arrivals[i])
            pairs += c["count"]
            retries += c["retries"]
            srv.release(c["request_id"])
            done += 1
        if nxt < len(reqs) and not backlog:
            time.sleep(max(0.0, min(2e-4, arrivals[nxt] - (time.monotonic() - t0))))
    return lat, time.monotonic() - t0, pairs, retries


def plain_run(C, built, reqs, arrivals, stats, fid, tid, res, h_res):
    """The same schedule, one request at a time through the plain per-batch
    form (count pass, scan, write pass)."""
    import time
    lat = np.zeros(len(reqs))
    t0 = time.monotonic()
    for i, (ti, w) in enumerate(reqs):
        wait = arrivals[i] - (time.monotonic() - t0)
        if wait > 0:
            time.sleep(wait)
        dq = C.BBox.from_host(w)
        C.query_into(built[ti][0], built[ti][1], dq, fid, tid, res, None, C.CRT_QUERY_PLAIN)
        h_res.copy_(res)
        r = C.read_result(h_res)
        assert r["count"] == stats[i], (r, stats[i])
        lat[i] = time.monotonic() - (t0 + arrivals[i])
    return lat, time.monotonic() - t0


def serving_leg(args, C, rank):
    import time

    import torch

    from curtree_b200.server import Server
    trees, reqs, gaps = serving_workload(args, rank)
    built = []
    for b in trees:
        d = C.BBox.from_host(b)
        rt = C.RTree(args.fanout)
        C.build_rtree(d, rt)
        built.append((rt, d))
    total_windows = sum(w.n for _, w in reqs)
    stats = []
    for ti, w in reqs:
        dq = C.BBox.from_host(w)
        stats.append(C.query_stats(built[ti][0], built[ti][1], dq)["hits"])
    cap = max(max(stats), 1)
    fid = torch.empty(cap, dtype=torch.int32, device="cuda")
    tid = torch.empty(cap, dtype=torch.int32, device="cuda")
    res = C.new_result_block()
    h_res = torch.empty(64, dtype=torch.uint8, pin_memory=True)

    srv = Server(arena_bytes=args.serve_arena_gb << 30, pairs_per_window=256.0)
    tids = [srv.add_tree(rt, d) for rt, d in built]
    # warm the device loop and the per-tree output estimates
    warm = min(8, len(reqs))
    serve_run(srv, tids, reqs[:warm], np.zeros(warm))
    summary = lambda lat, span: {
        "windows_per_s": total_windows / span, "requests_per_s": len(reqs) / span,
        "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "makespan_s": span}
    rates = []
    for rate in [float(x) for x in args.serve_rates.split(",")]:
        arrivals = gaps / rate
        lat, span, pairs, retries = serve_run(srv, tids, reqs, arrivals)
        assert pairs == sum(stats), (pairs, sum(stats))
        served = dict(summary(lat, span), pairs=int(pairs), retries=int(retries))
        lat_p, span_p = plain_run(C, built, reqs, arrivals, stats, fid, tid, res, h_res)
        plain = summary(lat_p, span_p)
        rates.append({"rate_req_s": rate, "offered_windows_per_s": total_windows / arrivals[-1],
                      "served": served, "plain": plain,
                      "served_vs_plain_windows_per_s": served["windows_per_s"] / plain["windows_per_s"],
                      "p99_served_le_plain": served["p99_ms"] <= plain["p99_ms"]})
        time.sleep(0.05)
    srv.close()
    return {"workload": f"trees {args.serve_trees} uniform boxes, fanout {args.fanout}; "
                        f"{len(reqs)} requests, Poisson arrivals, batch "
                        f"log-U[1, {args.serve_max_batch}] windows, side log-U[1e-5, 1e-1]",
            "windows": int(total_windows), "pairs": int(sum(stats)), "rates": rates}


def adversarial_leg(args, C, stream, dist, world, rank):
    """Road-like boxes (centres on 100 segments, Pareto long sides capped at
    0.5, aspect ratios up to 1e4) and a window mix of 50% points, 40% small
    windows and 10% windows over 1% of the domain.  Batched: every window
    through query_stream (one output buffer of 2^32 pairs, 32 GiB, reused;
    batches that overflow re-run smaller); pairs are counted and dropped, as
    a consumer that reduces them would.  Served: the first tenth of the windows as
    requests of 1-1000 windows arriving at 1k requests/s."""
    import time

    import torch

    from curtree_b200 import datasets as D
    from curtree_b200.server import Server
    b = D.road_boxes(args.adv_boxes, seed=5 + 1000 * rank)
    q = D.road_windows(args.adv_windows, seed=105 + 1000 * rank)
    d = C.BBox.from_host(b)
    del b
    rt = C.RTree(args.fanout)
    C.build_rtree(d, rt)
    dq = C.BBox.from_host(q)
    total = C.query_stats(rt, d, dq)["hits"]
    cap = C.query_capacity(1 << args.adv_buffer_log2)
    drop = lambda f, t, a: None
    warm = C.BBox(dq.xmin[:20_000], dq.ymin[:20_000], dq.xmax[:20_000], dq.ymax[:20_000],
                  dq.id[:20_000])
    C.query_stream(rt, d, warm, drop, capacity=cap)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st = C.query_stream(rt, d, dq, drop, capacity=cap, batch=1 << 16)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = reduce_max(e0.elapsed_time(e1), dist)
    assert st["pairs"] == total, (st, total)
    batched = {"windows_per_s": world * q.n / (ms / 1e3), "pairs_per_s": world * total / (ms / 1e3),
               "ms": ms, "pairs": int(total), "batches": st["batches"], "retries": st["retries"],
               "output_buffer_pairs": int(cap)}

    # served
    nserve = q.n // 10
    rng = np.random.default_rng(7 + rank)
    cuts = [0]
    while cuts[-1] < nserve:
        cuts.append(min(nserve, cuts[-1] + int(np.exp(rng.uniform(0, np.log(1000))))))
    reqs = list(zip(cuts[:-1], cuts[1:]))
    arrivals = np.cumsum(rng.exponential(1.0 / 1000.0, len(reqs)))
    srv = Server(arena_bytes=args.serve_arena_gb << 30, pairs_per_window=256.0)
    tree = srv.add_tree(rt, d)
    windows = [C.BBox(dq.xmin[a:e], dq.ymin[a:e], dq.xmax[a:e], dq.ymax[a:e], dq.id[a:e])
               for a, e in reqs]
    lat = np.zeros(len(reqs))
    backlog, ids = [], {}
    nxt = done = 0
    pairs = retries = 0
    t0 = time.monotonic()
    while done < len(reqs):
        now = time.monotonic() - t0
        if now > SERVE_DEADLINE_S:
            raise RuntimeError(f"serving run passed {SERVE_DEADLINE_S} s: {done} of {len(reqs)} done")
        while nxt < len(reqs) and arrivals[nxt] <= now:
            backlog.append(nxt)
            nxt += 1
        while backlog:
            rid = srv.submit(tree, windows[backlog[0]])
            if rid is None:
                break
            ids[rid] = backlog.pop(0)
        for c in srv.poll(max_out=256, wait_ms=0 if (backlog or nxt < len(reqs)) else 2):
            i = ids.pop(c["request_id"])
            if c["status"] != 0:
                raise RuntimeError(f"served request failed: {c}")
            lat[i] = c["complete_time_s"] - (t0 + arrivals[i])
            pairs += c["count"]
            retries += c["retries"]
            srv.release(c["request_id"])
            done += 1
        if nxt < len(reqs) and not backlog:
            time.sleep(max(0.0, min(2e-4, arrivals[nxt] - (time.monotonic() - t0))))
    span = time.monotonic() - t0
    srv.close()
    served_total = C.query_stats(rt, d, C.BBox(dq.xmin[:nserve], dq.ymin[:nserve], dq.xmax[:nserve],
                                                 dq.ymax[:nserve], dq.id[:nserve]))["hits"]
    assert pairs == served_total, (pairs, served_total)
    served = {"requests": len(reqs), "windows": int(nserve), "pairs": int(pairs),
              "windows_per_s": nserve / span, "p50_ms": float(np.percentile(lat, 50) * 1e3),
              "p99_ms": float(np.percentile(lat, 99) * 1e3), "retries": int(retries),
              "rate_req_s": 1000.0}
    rt.free()
    return {"workload": f"{args.adv_boxes // 1_000_000}M road boxes (100 segments, Pareto sides "
                        f"capped at 0.5, aspect up to 1e4), {args.adv_windows // 1000}k windows "
                        f"(50% points, 40% small, 10% over 1% of the domain), fanout {args.fanout}",
            "batched": batched, "served": served}


def ingest_leg(args, C, L, stream):
    """The reference's MBR text file read into device boxes: readMBR + box_h2d
    (src/utility.cpp:5-40, src/utility.cuh:42-66) against
    crt_read_mbr_csv_device, file in the page cache.  Each step is one call,
    timed on the host clock (the call returns once the boxes are on the
    device).  Beside it: the library's host loader (crt_read_mbr_csv, all
    host threads) followed by the copy to the device, and a pinned
    host-to-device copy of the same bytes, the link the device path rides."""
    import ctypes
    import tempfile
    import time

    import torch
    from curtree_b200 import _lib
    from curtree_b200 import datasets as D
    n = args.ingest_records
    boxes = D.uniform_boxes(n, seed=21)
    boxes.id[:] = np.random.default_rng(22).integers(-2**31, 2**31 - 1, n)
    text = D.mbr_csv_text(boxes)
    nbytes = len(text)
    sample = min(n, 500_000)
    cut = int(np.flatnonzero(np.frombuffer(text, np.uint8) == 10)[sample - 1]) + 1
    shm = "/dev/shm" if os.path.isdir("/dev/shm") else None
    fd, path = tempfile.mkstemp(suffix=".csv", dir=shm)
    fd2, path2 = tempfile.mkstemp(suffix=".csv", dir=shm)
    ref = None
    try:
        with os.fdopen(fd, "wb") as f:
            f.write(text)
        with os.fdopen(fd2, "wb") as f:
            f.write(text[:cut])
        del text
        # the reference's own readMBR (fscanf, one thread), built from its
        # sources, on the first records: the CPU baseline of this leg
        from oracle import oracle as O
        if O.ref_cpu_available():
            t0 = time.perf_counter()
            O.ref_read_mbr(path2, sample, 0.0)
            dt = time.perf_counter() - t0
            ref = {"value": sample / dt, "unit": "records/s", "cores": 1, "kind": "reference",
                   "sample": f"the first {sample} records, the reference's readMBR "
                             "(src/utility.cpp:5-40) compiled from its sources, host arrays only"}
        box = _lib.crt_bbox_f32()
        got = ctypes.c_int64(0)
        h = ctypes.c_void_p(stream.cuda_stream)

        def step():
            t0 = time.perf_counter()
            _lib.check(L.crt_read_mbr_csv_device(path.encode(), n, 0.0, ctypes.byref(box),
                                                 ctypes.byref(got), h), "read_mbr_csv_device")
            dt = time.perf_counter() - t0
            return dt

        L.crt_profile_enable(1)
        for _ in range(args.warmup):
            step()
            L.crt_bbox_free(ctypes.byref(box))
        profile_collect(None)
        launches0 = C.kernel_launches()
        secs = []
        for i in range(args.steps):
            secs.append(step())
            if i + 1 < args.steps:
                L.crt_bbox_free(ctypes.byref(box))
        launches = C.kernel_launches() - launches0
        parts = {k: profile_collect(k)[0] / args.steps
                 for k in ("ingest_stage", "ingest_lines", "ingest_emit", "ingest_parse")}
        profile_collect(None)
        L.crt_profile_enable(0)
        from curtree_b200.rtree import _d2h
        dev = [_d2h(p, n, np.float32) for p in (box.xmin, box.ymin, box.xmax, box.ymax)]
        dev_id = _d2h(box.id, n, np.int32)
        L.crt_bbox_free(ctypes.byref(box))

        # the same boxes as 28-byte binary records
        raw = D.mbr_bin_bytes(boxes)
        with open(path2, "wb") as f:
            f.write(raw)
        bin_bytes = len(raw)
        del raw
        bsecs = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            _lib.check(L.crt_read_mbr_bin_device(path2.encode(), n, 0.0, ctypes.byref(box),
                                                 ctypes.byref(got), h), "read_mbr_bin_device")
            if i >= args.warmup:
                bsecs.append(time.perf_counter() - t0)
            L.crt_bbox_free(ctypes.byref(box))
        binary = {"records_per_s": n / statistics.median(bsecs),
                  "ms_per_step": statistics.median(bsecs) * 1e3, "file_bytes": bin_bytes,
                  "gb_per_s": bin_bytes / statistics.median(bsecs) / 1e9,
                  "what": "crt_read_mbr_bin_device, 28-byte records of the same boxes"}

        # the host loader, then the copy of its arrays to the device
        host = [np.empty(n, np.float32) for _ in range(4)]
        host_id = np.empty(n, np.int32)
        hsecs = []
        for _ in range(2):
            t0 = time.perf_counter()
            _lib.check(L.crt_read_mbr_csv(path.encode(), n, 0.0, *[a.ctypes.data for a in host],
                                          host_id.ctypes.data, ctypes.byref(got)), "read_mbr_csv")
            d = [torch.from_numpy(a).cuda() for a in host + [host_id]]
            torch.cuda.synchronize()
            hsecs.append(time.perf_counter() - t0)
            del d
        identical = all(np.array_equal(a.view(np.uint32), b.view(np.uint32))
                        for a, b in zip(host, dev)) and np.array_equal(host_id, dev_id)

        # pinned host-to-device copy of the same number of bytes
        src = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
        dst = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        for _ in range(2):
            dst.copy_(src, non_blocking=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        h2d_gbs = 5 * nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9
        del src, dst
    finally:
        os.unlink(path)
        os.unlink(path2)
    sec = statistics.median(secs)
    kern_ms = parts["ingest_lines"] + parts["ingest_emit"] + parts["ingest_parse"]
    return {"metric": "mbr_records_per_s", "value": n / sec, "unit": "records/s",
            "text_gb_per_s": nbytes / sec / 1e9, "ms_per_step": sec * 1e3,
            "records": n, "text_bytes": nbytes, "bytes_per_record": nbytes / n,
            "phases_ms": parts, "gpu_kernels_ms": kern_ms,
            "gpu_text_gb_per_s": nbytes / (kern_ms / 1e3) / 1e9 if kern_ms else None,
            "gpu_launches": launches,
            "h2d_pinned_gb_per_s": h2d_gbs, "frac_of_h2d_copy": nbytes / sec / 1e9 / h2d_gbs,
            "host_loader": {"records_per_s": n / min(hsecs), "ms": min(hsecs) * 1e3,
                            "cores": os.cpu_count(),
                            "what": "crt_read_mbr_csv (host threads) + copy of the five arrays"},
            "speedup_vs_host_loader": min(hsecs) / sec, "identical_to_host_loader": bool(identical),
            "cpu_baseline": ref, "binary": binary,
            "workload": f"{n // 10**6}M records 'x1,y1,x2,y2,id,pid,nume' (6 fraction digits, "
                        "corners half swapped, random int32 ids), file in the page cache, "
                        "crt_read_mbr_csv_device(path, n, r=0)"}


def build_leg(args, C, L, hbm_peak, peak_kind, stream, dist, world):
    import torch
    from curtree_b200 import datasets as D
    n = args.build_boxes
    boxes = D.clustered_boxes(n, seed=2)
    d_in = C.BBox.from_host(boxes)
    del boxes
    f = 10
    rsz = C.tree_size(n, f)
    out = C.BBox.empty(n)
    rt = C.RTree(f)
    ts = [torch.empty(rsz, dtype=dt, device="cuda") for dt in [torch.float32] * 4 + [torch.int32] * 2]
    rt.s.xmin, rt.s.ymin, rt.s.xmax, rt.s.ymax, rt.s.pos, rt.s.len = [t.data_ptr() for t in ts]
    ci, co = d_in.c(), out.c()
    import ctypes
    from curtree_b200 import _lib

    def step():
        _lib.check(L.crt_build_into_f32(ctypes.byref(ci), ctypes.byref(co), ctypes.byref(rt.s),
                                        ctypes.c_void_p(stream.cuda_stream)), "build")

    L.crt_profile_enable(1)
    for _ in range(args.warmup):
        step()
    profile_collect(None)
    ms = timed(step, args.steps, stream)
    parts = {k: profile_collect(k)[0] / args.steps for k in ("encode", "sort_pass", "level")}
    profile_collect(None)
    L.crt_profile_enable(0)
    ms = reduce_max(ms, dist)
    kern_ms = sum(parts.values())
    b_build = 120 * n + 40 * rsz
    strict = 40 * n + 24 * rsz
    return {"metric": "build_boxes_per_s", "value": world * n / (ms / args.steps / 1e3),
            "unit": "boxes/s", "ms_per_step": ms / args.steps, "kernel_ms": kern_ms,
            "kernels_ms": parts, "fanout": f, "boxes": n, "r_sz": rsz,
            "workload": "100M clustered boxes (1000 Gaussians + 10% uniform, log-normal sides, "
                        "1% duplicates, 1% points), out-of-place crt_build_into_f32",
            "roofline": {"bound": "hbm", "achieved": b_build / (kern_ms / 1e3) / 1e9,
                         "peak": hbm_peak, "unit": "GB/s",
                         "frac": b_build / (kern_ms / 1e3) / 1e9 / hbm_peak, "traffic": None,
                         "peak_kind": peak_kind, "algorithmic_bytes": b_build,
                         "bytes_model": "120 B/box + 40 B/node",
                         "strict_io_frac": strict / (kern_ms / 1e3) / 1e9 / hbm_peak}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None

    if args.impl == "reference":
        if rank != 0:
            return
        from curtree_b200 import datasets as D
        boxes, windows = make_query_inputs(0, args.boxes, args.windows)
        vals = []
        samples = []
        per_step = max(2.0, args.cpu_seconds / 2)
        for i in range(args.warmup + args.steps):
            r = cpu_reference_rate(boxes, windows, per_step, rng_seed=11 + i)
            if i >= args.warmup:
                vals.append(r["value"])
                samples.append(r["sample"])
        v = statistics.median(vals)
        line = {"impl": "reference", "metric": "window_queries_per_s", "value": v,
                "unit": "windows/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": query_config(args),
                "cpu_baseline": {"value": v, "unit": "windows/s", "cores": r["cores"],
                                 "kind": r["kind"], "sample": samples[-1]},
                "e2e": {"value": v, "unit": "windows/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                 device_id=torch.device("cuda", local))
        dist = tdist
    out, boxes, windows = run_ours(args, rank, world, dist)
    skip = set(s for s in args.skip.split(",") if s)
    cpu = None
    if rank == 0 and world == 1 and "cpu" not in skip:
        cpu = cpu_reference_rate(boxes, windows, args.cpu_seconds)
    if rank == 0:
        p = out["persistent"]
        line = {"metric": "window_queries_per_s", "value": p["windows_per_s"], "unit": "windows/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": p["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": query_config(args),
                "roofline": out["roofline"], "cpu_baseline": cpu, "e2e": out.get("e2e"),
                "gpu_launches": out["gpu_launches"], "clocks": out["clocks"],
                "plain": out.get("plain"), "build": out.get("build"),
                "serving": out.get("serving"), "adversarial": out.get("adversarial"),
                "ingest": out.get("ingest"), "cpu_rtree": out.get("cpu_rtree"),
                "workload_stats": out["workload_stats"], "autotune": out.get("autotune"),
                "persistent_kernel_ms": p["kernel_ms"]}
        if "plain" in out:
            line["persistent_vs_plain"] = p["windows_per_s"] / out["plain"]["windows_per_s"]
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def query_config(args):
    return {"workload": f"{args.boxes // 10**6}M uniform boxes (side U[0,1e-3]) x "
                        f"{args.windows // 1000}k mixed windows (side log-U[1e-5,1e-1], half on "
                        f"box centres), fanout {args.fanout}, persistent graph-captured form",
            "boxes": args.boxes, "windows": args.windows, "fanout": args.fanout,
            "parallelism": "replicas (each GPU its own tree copy and window batch)",
            "l2": "inputs larger than L2 (box SoA 200 MB, pair output tens of GB); no flush"}


if __name__ == "__main__":
    main()
