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
    p.add_argument("--stage", type=int, default=2,
                   help="whole tree levels below the root staged in shared memory")
    p.add_argument("--window-warps", type=int, default=1, help="warps sharing one window")
    p.add_argument("--chunk", type=int, default=4096, help="output slots a warp reserves")
    p.add_argument("--sort-windows", type=int, default=1)
    p.add_argument("--autotune", type=int, default=1, help="pick fanout/warps/staging first (untimed)")
    p.add_argument("--autotune-windows", type=int, default=100_000)
    p.add_argument("--skip", default="",
                   help="comma list of legs to skip: build,e2e,plain,cpu,serve,adversarial,"
                        "ingest,config1")
    p.add_argument("--adv-boxes", type=int, default=50_000_000)
    p.add_argument("--adv-windows", type=int, default=2_000_000)
    p.add_argument("--adv-buffer-log2", type=int, default=32,
                   help="output buffer of the streamed adversarial leg: 2^k pairs")
    p.add_argument("--ingest-records", type=int, default=4_000_000,
                   help="records of the MBR text file the ingest leg reads")
    p.add_argument("--serve-trees", default="1000000,5000000,20000000,50000000")
    p.add_argument("--serve-requests", type=int, default=2000)
    p.add_argument("--serve-rates", default="1000,3000,10000,30000,100000",
                   help="comma list of Poisson arrival rates (requests/s)")
    p.add_argument("--serve-max-batch", type=int, default=100_000)
    p.add_argument("--serve-arena-gb", type=int, default=64)
    p.add_argument("--parity", type=int, default=1,
                   help="check the GPU's pairs against the oracle (untimed; per-window digests)")
    p.add_argument("--parity-windows", type=int, default=0,
                   help="windows of the headline batch the oracle checks (0: all at one GPU, "
                        "100k per rank under torchrun)")
    p.add_argument("--parity-adv-windows", type=int, default=50_000,
                   help="windows of the adversarial batch the oracle checks")
    p.add_argument("--parity-serve-every", type=int, default=8,
                   help="the oracle checks every k-th served request")
    p.add_argument("--reference-gpu", type=int, default=1,
                   help="reference arm: also time the reference's own GPU path (oracle/_ref)")
    p.add_argument("--detail", default="",
                   help="also write the full result (autotune table, every leg) to this JSON file")
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
def cpu_reference_rate(boxes, windows, seconds: float, rng_seed: int = 7, keep=False):
    """Windows/s of the reference's nested_loop_query over all host threads,
    on a sample of windows sized to about `seconds` of CPU work.  Falls back to
    the oracle's restatement when the reference build is absent.  keep: also
    return the sample's window indices with the per-window pair counts and
    digests of the pairs the reference emitted (for the parity check)."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    kind = "reference" if O.ref_cpu_available() else "port"
    rng = np.random.default_rng(rng_seed)

    def run(m):
        idx = np.sort(rng.choice(windows.n, size=min(m, windows.n), replace=False))
        q = windows.take(idx)
        if kind == "reference":
            c, h, pairs, t = O.ref_nested_loop_digest(q, boxes, idx.astype(np.int32), threads)
        else:
            t0 = time.perf_counter()
            c, h = O.nested_loop_stats(q, boxes, nthreads=threads)
            t = time.perf_counter() - t0
            h = None  # positional digests: not comparable with window indices
            pairs = int(c.sum())
        return q.n, t, int(pairs), (idx, c, h)

    n0, t0, _, _ = run(threads)
    m = int(max(threads, min(windows.n, n0 / max(t0, 1e-6) * seconds)))
    m = (m + threads - 1) // threads * threads
    n, t, pairs, kept = run(m)
    out = {"value": n / t, "unit": "windows/s", "cores": threads, "kind": kind,
           "sample": f"{n} of {windows.n} windows x {boxes.n} boxes, {t:.1f} s, {pairs} pairs"}
    return (out, kept) if keep else out


def cpu_rtree_rate(boxes, windows, seconds: float, rng_seed: int = 9):
    """Windows/s of a CPU R-tree on all host threads, as the reference's CPU
    check runs one (src/verify.hpp:35-95: Boost's rtree<value,
    quadratic<16>>, built by inserting the boxes one at a time, then queried
    window by window).  Boost is absent, so the index is the oracle's
    restatement of that algorithm (Guttman's quadratic split, 4-16 entries
    per node), built over the same boxes on one thread; the queries run on
    all host threads over a sample of windows sized to about `seconds` of
    CPU work, and their pairs are counted and digested."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(rng_seed)
    tree = O.QuadraticRTree(boxes)

    def run(m):
        idx = np.sort(rng.choice(windows.n, size=min(m, windows.n), replace=False))
        q = windows.take(idx)
        c, h, t = tree.query_stats(q, qid=idx.astype(np.int32), nthreads=threads)
        return q.n, t, int(c.sum()), (idx, c, h)

    n0, t0, _, _ = run(threads * 8)
    m = int(max(threads, min(windows.n, n0 / max(t0, 1e-6) * seconds)))
    m = (m + threads - 1) // threads * threads
    n, t, pairs, kept = run(m)
    build_s = tree.build_seconds
    tree.free()
    return {"value": n / t, "unit": "windows/s", "cores": threads, "kind": "port",
            "build_s": build_s,
            "sample": f"{n} of {windows.n} windows x {boxes.n} boxes, {t:.1f} s, {pairs} pairs",
            "what": "Guttman R-tree with the quadratic split, 4-16 entries per node, built by "
                    "inserting the boxes one at a time on one thread (the index of the "
                    "reference's Boost check, restated: Boost is absent); queries on all host "
                    "threads"}, kept


# ---------------------------------------------------------------------------
# parity at full size (untimed): per-window pair counts and order-independent
# digests of what the GPU wrote, against the oracle's tree query on the
# oracle's own build of the same boxes, and against the reference's own
# brute force (nested_loop_query) on the CPU baseline's sample.  This is the
# reference drivers' check (sort both pair vectors, compare them:
# src/rtree_test_frontier.cu:102-123) in a form that holds at 10^9-10^11 pairs.
# ---------------------------------------------------------------------------
def same_tree(h_tree, h_sorted, tr, sb) -> bool:
    keys = ("xmin", "ymin", "xmax", "ymax", "pos", "len")
    ok = all(np.array_equal(np.asarray(getattr(h_tree, k)).view(np.int32),
                            np.asarray(getattr(tr, k)).view(np.int32)) for k in keys)
    return bool(ok and all(np.array_equal(np.asarray(getattr(h_sorted, k)).view(np.int32),
                                          np.asarray(getattr(sb, k)).view(np.int32))
                           for k in ("xmin", "ymin", "xmax", "ymax", "id")))


def compare_digests(got_c, got_h, want_c, want_h) -> dict:
    bad = (got_c != want_c) | (got_h != want_h)
    return {"windows": int(want_c.size), "pairs": int(want_c.sum()),
            "counts_ok": bool(np.array_equal(got_c, want_c)),
            "digest_ok": bool(not bad.any()), "windows_differing": int(bad.sum())}


def sample_indices(n: int, m: int) -> np.ndarray:
    """All of [0, n) when m <= 0 or m >= n, else m indices spread evenly."""
    if m <= 0 or m >= n:
        return np.arange(n, dtype=np.int32)
    return np.unique(np.linspace(0, n - 1, m).astype(np.int64)).astype(np.int32)


def oracle_tree(boxes, fanout, rt, sorted_box):
    """The oracle's build of the same boxes and whether the GPU's tree and
    permuted boxes equal it bit for bit."""
    from oracle import oracle as O
    sb, tr = O.build(boxes, fanout)
    return sb, tr, same_tree(rt.to_host(), sorted_box.to_host(), tr, sb)


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


def per_step_ms(fn, steps, stream):
    """Device time of each of `steps` consecutive steps (events between them)."""
    import torch
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for i in range(steps):
        fn()
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    return [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]


def latency_summary(ms):
    return {"batches": len(ms), "p50_ms": float(np.percentile(ms, 50)),
            "p99_ms": float(np.percentile(ms, 99)), "max_ms": float(max(ms))}


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

    # ---- the reference's own small case through the drop-in calls, first:
    # measured like the reference's run of it, on a device whose memory pools
    # the large legs have not filled yet
    if "config1" not in skip and rank == 0:
        out["config1"] = config1_leg(args, C, stream)
        torch.cuda.empty_cache()
        out["small_windows"] = small_windows_leg(args, C, stream)
        torch.cuda.empty_cache()

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
        args.window_warps = tuned["warps_per_window"]
        args.chunk = tuned["chunk"]
        torch.cuda.empty_cache()
    out["autotune"] = None if tuned is None else {
        "chosen": {k: tuned[k] for k in ("fanout", "warps_per_cta", "stage_levels",
                                         "warps_per_window", "chunk", "ms")},
        "sample_windows": int(sample.n),
        "table": [{k: (round(v, 3) if isinstance(v, float) else v) for k, v in row.items()}
                  for row in tuned["table"]]}
    sorted_box, rt = C.build_into(d_in, args.fanout)
    del d_in
    d_win = C.BBox.from_host(windows)
    st = C.query_stats(rt, sorted_box, d_win)
    pairs, tested, tested_c = st["hits"], st["tested"], st["tested_contain"]
    cap = C.query_capacity(pairs, chunk=args.chunk)
    fid = torch.empty(cap, dtype=torch.int32, device="cuda")
    tid = torch.empty(cap, dtype=torch.int32, device="cuda")
    res = C.new_result_block()

    # ---- persistent form (graph plan) -------------------------------------
    L.crt_profile_enable(1)
    qopts = persistent_opts(args)
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
    # single-batch latency of the persistent form (untimed: each step alone)
    out["persistent"]["batch_latency"] = latency_summary(
        per_step_ms(plan.launch, max(args.steps, 20), stream))
    digests = {}
    if args.parity:
        # per-window counts and digests of the pairs the last launch wrote
        r = C.read_result(res)
        assert r["overflow"] == 0 and r["count"] == pairs, r
        dg = C.PairDigest(args.windows)
        dg.add(fid, tid, n=pairs)
        digests["persistent"] = dg.to_host()
        del dg
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
                        "kernel_ms": pk_ms / max(args.steps, 1),
                        "batch_latency": latency_summary(per_step_ms(plain, max(args.steps, 20),
                                                                     stream))}
        if args.parity:
            r = C.read_result(res)
            assert r["overflow"] == 0 and r["count"] == pairs, r
            dg = C.PairDigest(args.windows)
            dg.add(fid, tid, n=pairs)
            digests["plain"] = dg.to_host()
            del dg
        del offs

    # ---- parity of the headline batch against the oracle (untimed) -----------
    if args.parity:
        out["parity"] = parity_headline(args, boxes, windows, rt, sorted_box, digests, world)
        out["_digests"] = digests
        if dist is not None:  # every rank checked its own batch: all must agree
            import torch
            ok = torch.tensor([1 if out["parity"]["ok"] else 0], dtype=torch.int32, device="cuda")
            dist.all_reduce(ok, op=dist.ReduceOp.MIN)
            out["parity"]["ok"] = bool(ok.item())
            out["parity"]["ranks"] = world

    # ---- CPU R-tree on the same tree (rank 0 of a 1-GPU run) ------------------
    if "cpu" not in skip and rank == 0 and world == 1:
        try:
            out["cpu_rtree"], (idx, qc, qh) = cpu_rtree_rate(boxes, windows, args.cpu_seconds)
            if "persistent" in digests:
                c, h, _ = digests["persistent"]
                out["cpu_rtree"]["same_pairs_as_gpu"] = bool(np.array_equal(c[idx], qc) and
                                                             np.array_equal(h[idx], qh))
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


def parity_headline(args, boxes, windows, rt, sorted_box, digests, world):
    """The oracle's build of the headline boxes against the GPU's tree (bit
    for bit), and the oracle's tree query on its own tree against the
    per-window counts and digests of each GPU form's output: every window at
    one GPU, a spread sample per rank under torchrun."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    sb, tr, tree_ok = oracle_tree(boxes, args.fanout, rt, sorted_box)
    m = args.parity_windows if args.parity_windows > 0 else (0 if world == 1 else 100_000)
    idx = sample_indices(windows.n, m)
    q = windows if idx.size == windows.n else windows.take(idx)
    want = O.tree_query_stats(tr, sb, q, qid=idx)
    forms = {}
    for name, (c, h, bad) in digests.items():
        forms[name] = dict(compare_digests(c[idx], h[idx], want.counts, want.hashes),
                           pairs_outside_windows=bad,
                           total_pairs_ok=bool(int(c.sum()) == int(want.counts.sum()))
                           if idx.size == windows.n else None)
    ok = tree_ok and all(f["digest_ok"] and f["pairs_outside_windows"] == 0 for f in forms.values())
    return {"ok": bool(ok), "tree_identical": tree_ok, "windows_checked": int(idx.size),
            "pairs_checked": int(want.counts.sum()), "forms": forms,
            "oracle": "oracle/crt_oracle.c build + tree query (src/rtree_bulkload_thrust.cuh, "
                      "src/rtree_bfs_frontier.cuh semantics) on the host",
            "seconds": time.perf_counter() - t0}


def persistent_opts(args):
    """The persistent form's options the headline runs with (the autotuner's
    choice unless given)."""
    return {"warps_per_cta": args.warps, "stage_levels": args.stage,
            "sort_windows": args.sort_windows, "warps_per_window": args.window_warps,
            "chunk": args.chunk}


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
        C.query_into(rt, sorted_box, d_win, fid, tid, res, **persistent_opts(args))
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


def serve_run(srv, tids, reqs, arrivals, on_done=None):
    """Replays one arrival schedule through the server; returns latencies
    (arrival to completion), makespan, pairs and retries.  on_done(i, c) sees
    each completion before its release."""
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
            if on_done is not None:
                on_done(i, c)
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


def serving_parity(args, C, srv, tids, trees, built, reqs):
    """Every k-th request served again (untimed, as fast as admitted), each
    completion's pairs digested on the device by window, against the
    oracle's tree query on the oracle's own build of that tree."""
    import torch

    from oracle import oracle as O
    t0 = time.perf_counter()
    chk = list(range(0, len(reqs), max(1, args.parity_serve_every)))
    got = {}

    def digest(k, c):
        dg = C.PairDigest(reqs[chk[k]][1].n)
        dg.add_ptr(c["d_fid"], c["d_tid"], c["count"])
        torch.cuda.current_stream().synchronize()  # read before the release
        got[chk[k]] = dg.to_host()

    serve_run(srv, tids, [reqs[i] for i in chk], np.zeros(len(chk)), on_done=digest)
    oracle = {}
    trees_ok = True
    for ti in sorted({reqs[i][0] for i in chk}):
        sb, tr, ok = oracle_tree(trees[ti], args.fanout, built[ti][0], built[ti][1])
        oracle[ti] = (sb, tr)
        trees_ok = trees_ok and ok
    bad_req = windows = pairs = outside = 0
    for i in chk:
        ti, w = reqs[i]
        want = O.tree_query_stats(oracle[ti][1], oracle[ti][0], w)
        c, h, nb = got[i]
        outside += nb
        windows += w.n
        pairs += int(want.counts.sum())
        if not (np.array_equal(c, want.counts) and np.array_equal(h, want.hashes)):
            bad_req += 1
    return {"ok": bool(trees_ok and bad_req == 0 and outside == 0), "trees_identical": trees_ok,
            "requests_checked": len(chk), "requests_differing": bad_req, "windows_checked": windows,
            "pairs_checked": pairs, "pairs_outside_windows": outside,
            "sample": f"every {max(1, args.parity_serve_every)}th request, replayed untimed",
            "seconds": time.perf_counter() - t0}


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
    parity = serving_parity(args, C, srv, tids, trees, built, reqs) if args.parity else None
    srv.close()
    return {"parity": parity,
            "workload": f"trees {args.serve_trees} uniform boxes, fanout {args.fanout}; "
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
    # parity (untimed): the first windows (an i.i.d. sample of the mix) streamed
    # again with their pairs digested on the device
    m = min(q.n, max(0, args.parity_adv_windows)) if args.parity else 0
    adv_digest = None
    if m:
        dg = C.PairDigest(m)
        head = C.BBox(dq.xmin[:m], dq.ymin[:m], dq.xmax[:m], dq.ymax[:m], dq.id[:m])
        sp = C.query_stream(rt, d, head, lambda f, t, a: dg.add(f, t, window_base=a),
                            capacity=cap, batch=1 << 16)
        adv_digest = dg.to_host() + (sp,)
        del dg

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
    lat, span, pairs, retries = serve_run(srv, [tree], [(0, w) for w in windows], arrivals)
    # parity replay (untimed): the requests over the first windows again, as
    # fast as they are admitted, each one's pairs digested on completion
    served_dg = None
    if m:
        served_dg = C.PairDigest(nserve)
        first = [i for i, (a, e) in enumerate(reqs) if a < m]

        def digest(i, c):
            served_dg.add_ptr(c["d_fid"], c["d_tid"], c["count"], window_base=reqs[first[i]][0])
            torch.cuda.current_stream().synchronize()  # read before the release

        serve_run(srv, [tree], [(0, windows[i]) for i in first], np.zeros(len(first)),
                  on_done=digest)
    srv.close()
    served_total = C.query_stats(rt, d, C.BBox(dq.xmin[:nserve], dq.ymin[:nserve], dq.xmax[:nserve],
                                                 dq.ymax[:nserve], dq.id[:nserve]))["hits"]
    assert pairs == served_total, (pairs, served_total)
    served = {"requests": len(reqs), "windows": int(nserve), "pairs": int(pairs),
              "windows_per_s": nserve / span, "p50_ms": float(np.percentile(lat, 50) * 1e3),
              "p99_ms": float(np.percentile(lat, 99) * 1e3), "retries": int(retries),
              "rate_req_s": 1000.0}
    parity = None
    if m:
        from oracle import oracle as O
        t0p = time.perf_counter()
        sb, tr, tree_ok = oracle_tree(b, args.fanout, rt, d)
        want = O.tree_query_stats(tr, sb, q.take(np.arange(m)))
        bc, bh, bbad, sp = adv_digest
        batched_cmp = dict(compare_digests(bc, bh, want.counts, want.hashes),
                           pairs_outside_windows=bbad, retries=sp["retries"], batches=sp["batches"])
        sm = min(m, nserve)
        sc, sh, sbad = served_dg.to_host()
        served_cmp = dict(compare_digests(sc[:sm], sh[:sm], want.counts[:sm], want.hashes[:sm]),
                          pairs_outside_windows=sbad)
        parity = {"ok": bool(tree_ok and batched_cmp["digest_ok"] and served_cmp["digest_ok"]
                             and bbad == 0 and sbad == 0),
                  "tree_identical": tree_ok, "windows_checked": m,
                  "batched": batched_cmp, "served": served_cmp,
                  "sample": f"the first {m} windows (i.i.d. draws of the mix)",
                  "seconds": time.perf_counter() - t0p}
    rt.free()
    return {"workload": f"{args.adv_boxes // 1_000_000}M road boxes (100 segments, Pareto sides "
                        f"capped at 0.5, aspect up to 1e4), {args.adv_windows // 1000}k windows "
                        f"(50% points, 40% small, 10% over 1% of the domain), fanout {args.fanout}",
            "batched": batched, "served": served, "parity": parity}


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


def small_windows_case():
    """A batch both GPU paths answer: 10M uniform boxes (side U[0,1e-3]) and
    1M windows with side U[0,1e-3] (about 10 hits each), small enough for
    the reference's bfs_frontier, whose 32-window blocks stop past 1024
    frontier nodes (src/rtree_bfs_frontier.cuh:46-48)."""
    from curtree_b200 import datasets as D
    b = D.uniform_boxes(10_000_000, seed=3)
    return b, D.uniform_windows(1_000_000, seed=113, max_side=1e-3)


def small_windows_leg(args, C, stream, reps=3):
    """The small-windows batch through the drop-in calls (crt_build_f32 in
    place, crt_query_f32 allocating the pairs; fanout 10, the reference's
    default), median of `reps` builds and of `reps` queries after one
    untimed call of each, every window checked against the oracle's tree
    query on the oracle's own build."""
    import torch
    b, q = small_windows_case()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bms = []
    for r in range(reps + 1):  # the first build (device pool growth) is a warm-up
        if r:
            rt.free()
            del d
        d = C.BBox.from_host(b)
        rt = C.RTree(10)
        torch.cuda.synchronize()
        e0.record(stream)
        C.build_rtree(d, rt, stream)
        e1.record(stream)
        e1.synchronize()
        if r:
            bms.append(e0.elapsed_time(e1))
    build_ms = statistics.median(bms)
    dq = C.BBox.from_host(q)
    qms = []
    dg = None
    for r in range(reps + 1):
        torch.cuda.synchronize()
        e0.record(stream)
        pr = C.bfs_frontier(rt, d, dq, stream)
        e1.record(stream)
        e1.synchronize()
        if r:
            qms.append(e0.elapsed_time(e1))
        if r == reps and args.parity:
            g = C.PairDigest(q.n)
            g.add_ptr(pr.s.fid, pr.s.tid, pr.sz)
            dg = g.to_host()
        npairs = pr.sz
        pr.free()
    out = {"workload": "10M uniform boxes (side U[0,1e-3]) x 1M windows (side U[0,1e-3]), fanout 10; "
                       "crt_build_f32 + crt_query_f32 (drop-in)",
           "build_ms": build_ms, "query_ms": statistics.median(qms), "pairs": int(npairs),
           "windows_per_s": q.n / (statistics.median(qms) / 1e3)}
    if dg is not None:
        from oracle import oracle as O
        sb, tr, same = oracle_tree(b, 10, rt, d)
        want = O.tree_query_stats(tr, sb, q)
        cmp = compare_digests(dg[0], dg[1], want.counts, want.hashes)
        out["parity"] = dict(cmp, ok=bool(cmp["digest_ok"] and same and dg[2] == 0), tree_identical=same)
    rt.free()
    return out


def config1_leg(args, C, stream, reps=10):
    """The reference's own small case: 1M uniform boxes (side U[0,1e-3]),
    10k windows (side U[0,1e-2]), fanout 10, through the drop-in calls a
    reference caller makes (crt_build_f32 in place, crt_query_f32 allocating
    the pairs), median of `reps` calls each; every window's pairs checked
    against the reference's own brute force (nested_loop_query), as the
    reference's driver checks them (src/rtree_test_frontier.cu:97-123)."""
    import torch

    from curtree_b200 import datasets as D
    b = D.uniform_boxes(1_000_000, seed=1)
    q = D.uniform_windows(10_000, seed=101)
    bms, qms = [], []
    dg = None
    for r in range(reps + 1):
        d = C.BBox.from_host(b)
        rt = C.RTree(10)
        dq = C.BBox.from_host(q)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        C.build_rtree(d, rt, stream)
        e1.record(stream)
        e1.synchronize()
        b_ms = e0.elapsed_time(e1)
        e0.record(stream)
        pr = C.bfs_frontier(rt, d, dq, stream)
        e1.record(stream)
        e1.synchronize()
        if r:  # the first call of each is a warm-up
            bms.append(b_ms)
            qms.append(e0.elapsed_time(e1))
        if r == reps and args.parity:
            dg = C.PairDigest(q.n)
            dg.add_ptr(pr.s.fid, pr.s.tid, pr.sz)
            dg = dg.to_host()
        npairs = pr.sz
        pr.free()
        rt.free()
        del d, dq
    out = {"workload": "1M uniform boxes (side U[0,1e-3]) x 10k windows (side U[0,1e-2]), "
                       "fanout 10; crt_build_f32 + crt_query_f32 (drop-in)",
           "build_ms": statistics.median(bms), "query_ms": statistics.median(qms),
           "pairs": int(npairs), "calls": reps}
    if dg is not None:
        from oracle import oracle as O
        if O.ref_cpu_available():
            c, h, n, secs = O.ref_nested_loop_digest(q, b, np.arange(q.n, dtype=np.int32))
            cmp = compare_digests(dg[0], dg[1], c, h)
            out["parity"] = dict(cmp, ok=bool(cmp["digest_ok"] and dg[2] == 0),
                                 against="the reference's nested_loop_query on every window "
                                         f"({secs:.1f} s on {os.cpu_count()} host threads)")
    return out


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
    # the drop-in call as the reference's build_rtree is called (crt_build_f32:
    # in place, allocates the node arrays), on a fresh copy of the input each time
    work = C.BBox.empty(n)
    dms = []
    for _ in range(3):
        for dst, src in zip((work.xmin, work.ymin, work.xmax, work.ymax, work.id),
                            (d_in.xmin, d_in.ymin, d_in.xmax, d_in.ymax, d_in.id)):
            dst.copy_(src)
        rt2 = C.RTree(f)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        C.build_rtree(work, rt2, stream)
        e1.record(stream)
        e1.synchronize()
        dms.append(e0.elapsed_time(e1))
        rt2.free()
    del work
    kern_ms = sum(parts.values())
    b_build = 120 * n + 40 * rsz
    strict = 40 * n + 24 * rsz
    return {"metric": "build_boxes_per_s", "value": world * n / (ms / args.steps / 1e3),
            "unit": "boxes/s", "ms_per_step": ms / args.steps, "kernel_ms": kern_ms,
            "dropin_ms": statistics.median(dms),
            "kernels_ms": parts, "fanout": f, "boxes": n, "r_sz": rsz,
            "workload": "100M clustered boxes (1000 Gaussians + 10% uniform, log-normal sides, "
                        "1% duplicates, 1% points), out-of-place crt_build_into_f32",
            "roofline": {"bound": "hbm", "achieved": b_build / (kern_ms / 1e3) / 1e9,
                         "peak": hbm_peak, "unit": "GB/s",
                         "frac": b_build / (kern_ms / 1e3) / 1e9 / hbm_peak, "traffic": None,
                         "peak_kind": peak_kind, "algorithmic_bytes": b_build,
                         "bytes_model": "120 B/box + 40 B/node",
                         "strict_io_frac": strict / (kern_ms / 1e3) / 1e9 / hbm_peak}}


def reference_gpu_leg():
    """The reference's own GPU path (build_rtree + bfs_frontier compiled from
    its sources into oracle/_ref/ref_frontier, sm_100) on this GPU, timed
    with CUDA events by the runner: its small case (1M boxes x 10k windows),
    the 100M clustered build, and the 10M-box x 1M-window batch of this
    benchmark's headline, on which it stops at its frontier-queue limit."""
    import shutil

    from curtree_b200 import datasets as D
    from oracle import ref_gpu as R
    if not R.available("ref_frontier"):
        return {"unavailable": "oracle/_ref/ref_frontier was not built (the reference sources "
                               "were absent when build() ran)"}
    out = {"runner": "oracle/_ref/ref_frontier: the reference's build_rtree "
                     "(src/rtree_bulkload_thrust.cuh:62) and bfs_frontier "
                     "(src/rtree_bfs_frontier.cuh:292), unchanged, CUDA-event timed"}
    tmp = tempfile.mkdtemp(prefix="crt_ref_")
    try:
        cases = [("small", lambda: D.uniform_boxes(1_000_000, seed=1),
                  lambda b: D.uniform_windows(10_000, seed=101), 10, 5),
                 ("build_100M_clustered", lambda: D.clustered_boxes(100_000_000, seed=2),
                  None, 10, 3),
                 ("batched_10M_x_1M", lambda: D.uniform_boxes(10_000_000, seed=3),
                  lambda b: D.mixed_windows(1_000_000, b, seed=103), 10, 1),
                 ("small_windows_10M_x_1M", lambda: small_windows_case()[0],
                  lambda b: small_windows_case()[1], 10, 3)]
        for name, mk_b, mk_q, f, reps in cases:
            b = mk_b()
            bfile = os.path.join(tmp, name + "_b.crtb")
            b.write_crtb(bfile)
            qfile = None
            if mk_q is not None:
                q = mk_q(b)
                qfile = os.path.join(tmp, name + "_q.crtb")
                q.write_crtb(qfile)
                del q
            nb = b.n
            del b
            t0 = time.perf_counter()
            try:
                _, _, pairs, info = R.run("ref_frontier", "query" if qfile else "build", bfile, qfile,
                                          f, os.path.join(tmp, name), reps=reps, timeout=600,
                                          want_pairs=False)
                rec = {"boxes": nb, "fanout": f, "build_ms": statistics.median(info["build_ms"]),
                       "build_boxes_per_s": nb / (statistics.median(info["build_ms"]) / 1e3)}
                if info.get("query_ms"):
                    rec["query_ms"] = statistics.median(info["query_ms"])
                if "pairs" in info:
                    rec["pairs"] = info["pairs"]
            except R.RefRunFailed as e:
                tail = [ln for ln in (e.stdout + e.stderr).splitlines() if ln.strip()][-2:]
                rec = {"boxes": nb, "fanout": f, "failed": f"exit {e.rc}", "output_tail": tail}
            rec["wall_s"] = time.perf_counter() - t0
            out[name] = rec
            for x in os.listdir(tmp):
                pth = os.path.join(tmp, x)
                shutil.rmtree(pth) if os.path.isdir(pth) else os.remove(pth)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


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
        if args.reference_gpu:
            try:
                line["reference_gpu"] = reference_gpu_leg()
            except Exception as e:  # a side record: report it, keep the line
                line["reference_gpu"] = {"error": f"{type(e).__name__}: {e}"}
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
        cpu, (idx, rc, rh) = cpu_reference_rate(boxes, windows, args.cpu_seconds, keep=True)
        dg = out.pop("_digests", {})
        if rh is not None and "persistent" in dg and out.get("parity"):
            c, h, _ = dg["persistent"]
            cmp = compare_digests(c[idx], h[idx], rc, rh)
            out["parity"]["reference_brute_force"] = dict(
                cmp, what="the reference's own nested_loop_query (src/utility.h:22-45, compiled "
                          "from its sources) on the CPU baseline's sample, against the persistent "
                          "form's digests")
            out["parity"]["ok"] = bool(out["parity"]["ok"] and cmp["digest_ok"])
    out.pop("_digests", None)
    if rank == 0:
        p = out["persistent"]
        detail = {"persistent": p, "plain": out.get("plain"), "build": out.get("build"),
                  "serving": out.get("serving"), "adversarial": out.get("adversarial"),
                  "ingest": out.get("ingest"), "cpu_rtree": out.get("cpu_rtree"),
                  "workload_stats": out["workload_stats"], "autotune": out.get("autotune"),
                  "parity": out.get("parity"), "e2e": out.get("e2e"), "roofline": out["roofline"],
                  "config1": out.get("config1"), "small_windows": out.get("small_windows")}
        if args.detail:
            with open(args.detail, "w") as f:
                json.dump(detail, f, indent=1)
        print("detail: " + json.dumps(detail), file=sys.stderr, flush=True)
        line = {"metric": "window_queries_per_s", "value": p["windows_per_s"], "unit": "windows/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": p["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": query_config(args),
                "roofline": out["roofline"], "cpu_baseline": cpu, "e2e": out.get("e2e"),
                "gpu_launches": out["gpu_launches"], "clocks": out["clocks"],
                "persistent_kernel_ms": p["kernel_ms"]}
        line.update(compact_legs(out))
        if "plain" in out:
            line["persistent_vs_plain"] = p["windows_per_s"] / out["plain"]["windows_per_s"]
            line["batch_latency_ms"] = {
                "persistent": {k: round(v, 3) for k, v in p["batch_latency"].items()},
                "plain": {k: round(v, 3) for k, v in out["plain"]["batch_latency"].items()}}
        line["parity"] = compact_parity(out)
        print(json.dumps(line), flush=True)
        failed = [k for k, v in line["parity"].items() if isinstance(v, dict) and v.get("ok") is False]
        if failed:
            print(f"parity FAILED: {failed}", file=sys.stderr, flush=True)
            sys.exit(3)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _r(x, nd=3):
    return None if x is None else round(float(x), nd)


def compact_legs(out):
    """The sub-legs in a few keys each, so the end of the line carries them;
    the full figures go to the detail record."""
    o = {}
    cr = out.get("cpu_rtree")
    if cr and "value" in cr:
        o["cpu_rtree"] = {"windows_per_s": _r(cr["value"], 1), "build_s": _r(cr["build_s"], 2),
                          "same_pairs_as_gpu": cr.get("same_pairs_as_gpu")}
    a = out.get("autotune")
    if a:
        o["autotune"] = {"chosen": a["chosen"], "rows": len(a["table"]),
                         "sample_windows": a["sample_windows"]}
    g = out.get("ingest")
    if g:
        o["ingest"] = {"records_per_s": _r(g["value"], 0), "ms": _r(g["ms_per_step"]),
                       "gpu_kernels_ms": _r(g["gpu_kernels_ms"]),
                       "speedup_vs_host_loader": _r(g["speedup_vs_host_loader"], 1),
                       "identical_to_host_loader": g["identical_to_host_loader"],
                       "binary_records_per_s": _r(g["binary"]["records_per_s"], 0)}
    v = out.get("adversarial")
    if v:
        b, sv = v["batched"], v["served"]
        o["adversarial"] = {"batched_pairs_per_s": _r(b["pairs_per_s"], 0), "batched_ms": _r(b["ms"], 1),
                            "pairs": b["pairs"], "retries": b["retries"],
                            "served_p50_ms": _r(sv["p50_ms"], 2), "served_p99_ms": _r(sv["p99_ms"], 2),
                            "served_retries": sv["retries"]}
    sv = out.get("serving")
    if sv:
        o["serving"] = [{"rate": int(r["rate_req_s"]), "served_wps": _r(r["served"]["windows_per_s"], 0),
                         "plain_wps": _r(r["plain"]["windows_per_s"], 0),
                         "ratio": _r(r["served_vs_plain_windows_per_s"], 2),
                         "p99_ms": [_r(r["served"]["p99_ms"], 1), _r(r["plain"]["p99_ms"], 1)]}
                        for r in sv["rates"]]
    if out.get("plain"):
        o["plain_windows_per_s"] = _r(out["plain"]["windows_per_s"], 0)
    c1 = out.get("config1")
    if c1:
        o["config1"] = {"build_ms": _r(c1["build_ms"]), "query_ms": _r(c1["query_ms"]),
                        "pairs": c1["pairs"]}
    sw = out.get("small_windows")
    if sw:
        o["small_windows"] = {"build_ms": _r(sw["build_ms"]), "query_ms": _r(sw["query_ms"]),
                              "pairs": sw["pairs"]}
    bd = out.get("build")
    if bd:
        o["build"] = {"boxes_per_s": _r(bd["value"], 0), "ms_per_step": _r(bd["ms_per_step"]),
                      "dropin_ms": _r(bd["dropin_ms"]),
                      "kernels_ms": {k: _r(x) for k, x in bd["kernels_ms"].items()},
                      "roofline_frac": _r(bd["roofline"]["frac"]),
                      "strict_io_frac": _r(bd["roofline"]["strict_io_frac"])}
    return o


def compact_parity(out):
    p = {}
    h = out.get("parity")
    if h:
        p["headline"] = {"ok": h["ok"], "tree_identical": h["tree_identical"],
                         "windows_checked": h["windows_checked"], "pairs_checked": h["pairs_checked"],
                         "forms_digest_ok": {k: f["digest_ok"] for k, f in h["forms"].items()}}
        rb = h.get("reference_brute_force")
        if rb:
            p["reference_brute_force"] = {"ok": rb["digest_ok"], "windows": rb["windows"],
                                          "pairs": rb["pairs"]}
    c1 = (out.get("config1") or {}).get("parity")
    if c1:
        p["config1"] = {"ok": c1["ok"], "windows": c1["windows"], "pairs": c1["pairs"]}
    sw = (out.get("small_windows") or {}).get("parity")
    if sw:
        p["small_windows"] = {"ok": sw["ok"], "windows": sw["windows"], "pairs": sw["pairs"]}
    v = (out.get("adversarial") or {}).get("parity")
    if v:
        p["adversarial"] = {"ok": v["ok"], "tree_identical": v["tree_identical"],
                            "windows_checked": v["windows_checked"],
                            "pairs_checked": v["batched"]["pairs"],
                            "batched_ok": v["batched"]["digest_ok"], "served_ok": v["served"]["digest_ok"]}
    sv = (out.get("serving") or {}).get("parity")
    if sv:
        p["serving"] = {"ok": sv["ok"], "trees_identical": sv["trees_identical"],
                        "requests_checked": sv["requests_checked"],
                        "windows_checked": sv["windows_checked"], "pairs_checked": sv["pairs_checked"]}
    return p


def query_config(args):
    return {"workload": f"{args.boxes // 10**6}M uniform boxes (side U[0,1e-3]) x "
                        f"{args.windows // 1000}k mixed windows (side log-U[1e-5,1e-1], half on "
                        f"box centres), fanout {args.fanout}, persistent graph-captured form",
            "boxes": args.boxes, "windows": args.windows, "fanout": args.fanout,
            "parallelism": "replicas (each GPU its own tree copy and window batch)",
            "l2": "inputs larger than L2 (box SoA 200 MB, pair output tens of GB); no flush"}


if __name__ == "__main__":
    main()
