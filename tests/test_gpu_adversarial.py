"""Adversarial geometry on the GPU (reduced instance of the road workload):
2M boxes on 100 line segments with Pareto long sides (capped at 0.5) and
aspect ratios up to 1e4; 20k windows, half degenerate points, 40% small and
10% covering more than 1% of the domain (about 1.5e8 pairs in all).  The
streamed batch form (fixed output buffer, overflow-and-retry) and the served
form give every window the oracle's pair count and pair digest."""
import time

import numpy as np
import pytest

from curtree_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def _s64(x: int) -> int:
    return x - (1 << 64) if x >= 1 << 63 else x


def _lsr(t, k: int):
    # logical right shift of int64 tensors
    return (t >> k) & ((1 << (64 - k)) - 1)


def mix64_torch(z):
    """The oracle's per-pair digest (splitmix64 finaliser) on int64 tensors
    with wrap-around arithmetic."""
    z = z + _s64(0x9E3779B97F4A7C15)
    z = (z ^ _lsr(z, 30)) * _s64(0xBF58476D1CE4E5B9)
    z = (z ^ _lsr(z, 27)) * _s64(0x94D049BB133111EB)
    return z ^ _lsr(z, 31)


class Digest:
    """Per-window pair counts and digests accumulated on the device."""

    def __init__(self, nq):
        import torch
        self.counts = torch.zeros(nq, dtype=torch.int64, device="cuda")
        self.hashes = torch.zeros(nq, dtype=torch.int64, device="cuda")

    def add(self, fid, tid, first=0):
        import torch
        if fid.numel() == 0:
            return
        t = tid.long() + first
        z = (t << 32) | (fid.long() & 0xFFFFFFFF)
        self.counts.index_add_(0, t, torch.ones_like(t))
        self.hashes.index_add_(0, t, mix64_torch(z))

    def check(self, want):
        c = self.counts.cpu().numpy()
        h = self.hashes.cpu().numpy().view(np.uint64)
        assert np.array_equal(c, want.counts)
        assert np.array_equal(h, want.hashes)


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    b = D.road_boxes(2_000_000, seed=5, chunk=2_000_000)
    q = D.road_windows(20_000, seed=105)
    d = C.BBox.from_host(b)
    rt = C.RTree(16)
    C.build_rtree(d, rt)
    sb, t = O.build(b, 16)
    mine = rt.to_host()
    for k in ("xmin", "ymin", "xmax", "ymax", "pos", "len"):
        assert np.array_equal(np.asarray(getattr(mine, k)).view(np.int32),
                              np.asarray(getattr(t, k)).view(np.int32)), k
    want = O.tree_query_stats(t, sb, q)
    assert want.counts.sum() > 50_000_000, "the big windows must dominate the output"
    return C, b, q, d, rt, want


def test_digest_matches_oracle_digest(env):
    """The device digest equals the oracle's on a known pair list."""
    import torch
    rng = np.random.default_rng(3)
    fid = rng.integers(-2**31, 2**31, 10_000).astype(np.int32)
    tid = rng.integers(0, 100, 10_000).astype(np.int32)
    dg = Digest(100)
    dg.add(torch.from_numpy(fid).cuda(), torch.from_numpy(tid).cuda())
    c, h = O.pair_hashes(fid, tid, 100)
    assert np.array_equal(dg.counts.cpu().numpy(), c)
    assert np.array_equal(dg.hashes.cpu().numpy().view(np.uint64), h)


@pytest.mark.parametrize("mode", ["persistent", "plain"])
def test_streamed_batches_with_overflow_and_retry(env, mode):
    C, b, q, d, rt, want = env
    m = C.CRT_QUERY_PERSISTENT if mode == "persistent" else C.CRT_QUERY_PLAIN
    cap = C.query_capacity(4_000_000, m)  # room for 4M pairs a batch
    dq = C.BBox.from_host(q)
    dg = Digest(q.n)
    st = C.query_stream(rt, d, dq, dg.add, capacity=cap, batch=1 << 16, mode=m)
    assert st["retries"] > 0 and st["batches"] > 10
    assert st["pairs"] == int(want.counts.sum())
    dg.check(want)


def test_served_requests(env):
    """Requests of 1-500 windows from the same mix, served with a per-window
    output estimate far too low for the big windows: results re-run with
    their exact size and equal the oracle's."""
    C, b, q, d, rt, want = env
    from curtree_b200.server import Server
    srv = Server(arena_bytes=4 << 30, pairs_per_window=1.0, output_slack=1.0)
    tree = srv.add_tree(rt, d)
    rng = np.random.default_rng(9)
    cuts = [0]
    while cuts[-1] < q.n:
        cuts.append(min(q.n, cuts[-1] + int(np.exp(rng.uniform(0, np.log(500))))))
    reqs = list(zip(cuts[:-1], cuts[1:]))
    dg = Digest(q.n)
    ids, queue, done, retries = {}, list(range(len(reqs))), 0, 0
    t0 = time.monotonic()
    while done < len(reqs) and time.monotonic() - t0 < 300:
        while queue:
            a, e = reqs[queue[0]]
            w = D.HostBoxes(q.xmin[a:e], q.ymin[a:e], q.xmax[a:e], q.ymax[a:e], q.id[a:e])
            rid = srv.submit(tree, w)
            if rid is None:
                break
            ids[rid] = queue.pop(0)
        for c in srv.poll(max_out=64, wait_ms=5):
            i = ids.pop(c["request_id"])
            assert c["status"] == 0, c
            fid, tid = Server.pairs(c)
            import torch
            dg.add(torch.from_numpy(fid).cuda(), torch.from_numpy(tid).cuda(), reqs[i][0])
            retries += c["retries"]
            srv.release(c["request_id"])
            done += 1
    assert done == len(reqs), "requests did not complete"
    assert retries > 0
    dg.check(want)
    assert srv.close() == 0
