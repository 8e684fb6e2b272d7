"""Serving loop on the GPU (continuous batching through one persistent kernel):
each request's result is the same in the mix as alone, requests admitted by
HBM footprint, undersized outputs re-run with their exact size, and a
device-side wait that runs out is reported as a status without harming the
context."""
import time

import numpy as np
import pytest

from curtree_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    from curtree_b200.server import Server
    trees = []
    for i, (n, f) in enumerate([(200_000, 10), (500_000, 16), (1_000_000, 8)]):
        b = D.uniform_boxes(n, seed=70 + i)
        d = C.BBox.from_host(b)
        rt = C.RTree(f)
        C.build_rtree(d, rt)
        sb, t = O.build(b, f)
        trees.append({"rt": rt, "d": d, "sb": sb, "t": t, "f": f})
    return C, Server, trees


def make_requests(trees, n_req, seed, max_windows=3000):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n_req):
        ti = int(rng.integers(0, len(trees)))
        nq = int(np.exp(rng.uniform(0, np.log(max_windows))))
        w = D.mixed_windows(nq, trees[ti]["sb"], seed=1000 * seed + i, lo=1e-5, hi=3e-2)
        reqs.append((ti, w))
    return reqs


def expected(trees, ti, w):
    t = trees[ti]
    return O.canonical_pairs(*O.tree_query_pairs(t["t"], t["sb"], w))


def run_all(srv, tree_ids, reqs, timeout_s=120):
    ids = {}
    done = {}
    queue = list(range(len(reqs)))
    t0 = time.monotonic()
    while (queue or len(done) < len(reqs)) and time.monotonic() - t0 < timeout_s:
        while queue:
            i = queue[0]
            rid = srv.submit(tree_ids[reqs[i][0]], reqs[i][1])
            if rid is None:
                break
            ids[rid] = i
            queue.pop(0)
        for c in srv.poll(max_out=64, wait_ms=5):
            i = ids[c["request_id"]]
            done[i] = (c, srv.pairs(c))
            srv.release(c["request_id"])
    assert not queue and len(done) == len(reqs), "requests did not complete"
    return done


def setup_server(C, Server, trees, **kw):
    srv = Server(**kw)
    ids = [srv.add_tree(t["rt"], t["d"]) for t in trees]
    return srv, ids


def test_results_same_alone_and_in_the_mix(env):
    C, Server, trees = env
    srv, ids = setup_server(C, Server, trees, arena_bytes=2 << 30)
    reqs = make_requests(trees, 80, seed=1)
    done = run_all(srv, ids, reqs)
    for i, (ti, w) in enumerate(reqs):
        c, (fid, tid) = done[i]
        assert c["status"] == 0
        got = O.canonical_pairs(fid, tid)
        want = expected(trees, ti, w)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), i
        # alone: the same request through the plain per-batch form
        dq = C.BBox.from_host(w)
        pf, pt, _ = C.query(trees[ti]["rt"], trees[ti]["d"], dq, mode=C.CRT_QUERY_PLAIN)
        alone = O.canonical_pairs(pf.cpu().numpy(), pt.cpu().numpy())
        assert np.array_equal(alone[0], got[0]) and np.array_equal(alone[1], got[1])
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["arena_used"] == 0
    assert srv.close() == 0


def test_tree_with_boxes_not_ordinary(env):
    """A served tree holding inverted boxes and NaN corners: the serving
    kernel must not take the containment shortcut on it (the predicate can
    reject such a box under a contained MBR); results equal the oracle's."""
    C, Server, _ = env
    b = D.uniform_boxes(200_000, seed=79)
    k = np.random.default_rng(79).choice(b.n, 400, replace=False)
    b.xmin[k[:200]], b.xmax[k[:200]] = b.xmax[k[:200]].copy(), b.xmin[k[:200]].copy()
    b.ymax[k[200:]] = np.nan
    d = C.BBox.from_host(b)
    rt = C.RTree(10)
    C.build_rtree(d, rt)
    sb, t = O.build(b, 10)
    tree = [{"rt": rt, "d": d, "sb": sb, "t": t, "f": 10}]
    srv, ids = setup_server(C, Server, tree, arena_bytes=1 << 30)
    reqs = [(0, D.mixed_windows(400, None, seed=790 + i, lo=1e-2, hi=0.5)) for i in range(4)]
    done = run_all(srv, ids, reqs)
    for i, (ti, w) in enumerate(reqs):
        c, (fid, tid) = done[i]
        assert c["status"] == 0
        got = O.canonical_pairs(fid, tid)
        want = expected(tree, ti, w)
        assert len(want[0]) > 0
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), i
    assert srv.close() == 0


def test_client_kernels_while_the_loop_runs(env):
    """A kernel the client launches while the device loop is up (held up
    1 s after its last request by idle_ms) may queue behind the loop when its
    stream shares a hardware queue with the loop's; the loop still stops on
    time -- the host's stop flag and error word need no CUDA call -- so the
    kernel runs by then, and the loop ends without a timeout.  Before, the
    dispatcher's own copies waited behind that kernel, the loop ran on until
    its bounded wait (device_wait_us, 20 s here) ended it with
    CRT_ERR_DEVICE_TIMEOUT."""
    import torch
    C, Server, trees = env
    srv, ids = setup_server(C, Server, trees, arena_bytes=1 << 30, idle_ms=1000,
                            device_wait_us=20_000_000)
    w = D.mixed_windows(2000, trees[2]["sb"], seed=91, lo=1e-4, hi=3e-2)
    rid = srv.submit(ids[2], w)
    cs = []
    t0 = time.monotonic()
    while not cs and time.monotonic() - t0 < 30:
        cs = srv.poll(wait_ms=10)
    assert cs and cs[0]["status"] == 0
    got = O.canonical_pairs(*Server.pairs(cs[0]))
    want = expected(trees, 2, w)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    x = torch.ones(1 << 22, device="cuda")
    t1 = time.monotonic()
    for _ in range(20):
        x = x * 1.0001 + 1.0
    s = float(x.sum().item())  # waits for this stream only
    elapsed = time.monotonic() - t1
    assert s > 0 and elapsed < 3.0, elapsed
    srv.release(rid)
    assert srv.close() == 0


def test_overflow_and_retry(env):
    C, Server, trees = env
    srv, ids = setup_server(C, Server, trees, pairs_per_window=0.01, output_slack=0.01)
    reqs = make_requests(trees, 25, seed=2)
    done = run_all(srv, ids, reqs)
    retried = sum(done[i][0]["retries"] for i in done)
    assert retried > 0 and srv.stats()["retried"] == retried
    for i, (ti, w) in enumerate(reqs):
        got = O.canonical_pairs(*done[i][1])
        want = expected(trees, ti, w)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), i
    srv.close()


def test_admission_by_footprint(env):
    C, Server, trees = env
    # the windows alone (16 B each, 2.4 MB) leave room for one request at a time
    srv, ids = setup_server(C, Server, trees, arena_bytes=4 << 20, pairs_per_window=1.0)
    w = D.mixed_windows(150_000, trees[0]["sb"], seed=77, lo=1e-5, hi=1e-4)
    a = srv.submit(ids[0], w)
    assert a is not None
    b = srv.submit(ids[0], w)
    assert b is None, "a second request must wait for arena space"
    cs = []
    t0 = time.monotonic()
    while not cs and time.monotonic() - t0 < 30:
        cs = srv.poll(wait_ms=10)
    assert cs and cs[0]["request_id"] == a
    srv.release(a)
    assert srv.submit(ids[0], w) is not None
    srv.close()


def test_device_wait_timeout_is_reported(env):
    """The idle device loop's bounded wait runs out (no work is published and
    the host does not stop it for 10 s): the kernel records
    CRT_ERR_DEVICE_TIMEOUT and returns; the host reads the status and later
    requests still run."""
    C, Server, trees = env
    srv, ids = setup_server(C, Server, trees, idle_ms=10_000, device_wait_us=5_000)
    w = D.mixed_windows(500, trees[1]["sb"], seed=78, lo=1e-5, hi=1e-2)
    rid = srv.submit(ids[1], w)
    cs = []
    t0 = time.monotonic()
    while not cs and time.monotonic() - t0 < 30:
        cs = srv.poll(wait_ms=10)
    assert cs and cs[0]["status"] == 0
    srv.release(rid)
    time.sleep(0.3)
    assert srv.stats()["device_status"] == C._lib.CRT_ERR_DEVICE_TIMEOUT
    # the context is intact: another request runs to completion, exactly
    rid = srv.submit(ids[1], w)
    cs = []
    t0 = time.monotonic()
    while not cs and time.monotonic() - t0 < 30:
        cs = srv.poll(wait_ms=10)
    assert cs and cs[0]["status"] == 0
    got = O.canonical_pairs(*Server.pairs(cs[0]))
    want = expected(trees, 1, w)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    srv.release(rid)
    srv.close()


def _wait_for(srv, rid, timeout_s=30.0):
    t0 = time.monotonic()
    while time.monotonic() - t0 < timeout_s:
        for c in srv.poll(max_out=16, wait_ms=10):
            if c["request_id"] == rid:
                return c
            srv.release(c["request_id"])
    raise AssertionError(f"request {rid} did not complete within {timeout_s} s")


def test_rerun_after_fragmentation(env):
    """A re-run whose exact output fits the arena only as one block with its
    windows: the request's window block sits in the middle of the arena
    (after a large request that completed and was released), so neither hole
    beside it can hold the output.  The re-run moves its windows out and back
    and completes with the oracle's pairs; a re-run that can never fit ends
    with CRT_ERR_OOM.  Both within 30 s, with the device loop idle between."""
    C, Server, trees = env
    t = trees[0]
    arena = 32 << 20
    srv, ids = setup_server(C, Server, trees, arena_bytes=arena, pairs_per_window=0.001,
                            output_slack=0.01)
    # R0: 1M windows far outside the tree (no hits): a 16 MB window block at
    # the start of the arena
    n0 = 1_000_000
    far = np.full(n0, -2.0e6, np.float32)
    r0 = D.HostBoxes(far, far, far + 1, far + 1, np.arange(n0, dtype=np.int32))
    # R1: windows whose exact output (2.6M-3.6M pairs) is larger than either
    # hole left around R1's windows once R0 is released
    pool = D.uniform_windows(20_000, seed=79, max_side=0.09)
    counts = C.query_stats(t["rt"], t["d"], C.BBox.from_host(pool),
                           per_window=True)["per_window_hits"].cpu().numpy()
    cum = np.cumsum(counts)
    k = int(np.searchsorted(cum, 3_000_000)) + 1
    assert 2_600_000 <= cum[k - 1] <= 3_600_000
    r1 = pool.take(np.arange(k))
    need = int(cum[k - 1])
    assert need * 8 > arena // 2 and need * 8 + 16 * k + 512 < arena
    a = srv.submit(ids[0], r0)
    b = srv.submit(ids[0], r1)
    assert a is not None and b is not None
    t0 = time.monotonic()
    ca = _wait_for(srv, a)
    assert ca["status"] == 0 and ca["count"] == 0
    srv.release(a)
    cb = _wait_for(srv, b)
    assert cb["status"] == 0 and cb["retries"] >= 1 and cb["count"] == need
    got = O.canonical_pairs(*Server.pairs(cb))
    want = expected(trees, 0, r1)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    srv.release(b)
    # a re-run whose exact output is larger than the whole arena fails cleanly
    k2 = int(np.searchsorted(cum, 6_000_000)) + 1
    r2 = pool.take(np.arange(k2))
    c = srv.submit(ids[0], r2)
    assert c is not None
    cc = _wait_for(srv, c)
    assert cc["status"] == C._lib.CRT_ERR_OOM and cc["count"] == int(cum[k2 - 1])
    srv.release(c)
    assert time.monotonic() - t0 < 30
    st = srv.stats()
    assert st["arena_used"] == 0 and st["retried"] >= 2
    assert srv.close() == 0
