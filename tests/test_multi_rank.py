"""The N-GPU benchmark path on CPU ranks (gloo, world size 2): replicas only,
so every rank builds the same tree from the same boxes, queries its own
window batch (weak scaling), and the reported step time is the maximum over
ranks.  No collective touches the data path."""
import hashlib
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _digest(b):
    h = hashlib.sha1()
    for a in (b.xmin, b.ymin, b.xmax, b.ymax, b.id):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        step_ms = bench.reduce_max(10.0 + 5 * rank, dist, "cpu")
        boxes, windows = bench.make_query_inputs(rank, 2000, 300)
        out.put((rank, step_ms, _digest(boxes), _digest(windows)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks_replicas_and_max_step_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, b0, w0), (r1, ms1, b1, w1) = res
    assert ms0 == ms1 == 15.0          # max over ranks on every rank
    assert b0 == b1                    # the same tree everywhere (replica)
    assert w0 != w1                    # each rank its own windows (weak scaling)


def _parity_worker(rank, world, port, out):
    """One replica rank: the library's host-side tree sizing, the oracle's
    build of this rank's replica, and the bench's parity check of this rank's
    window batch (the oracle's own per-window digests stand in for the GPU's,
    as no GPU is used here); then the parity flags reduced over the ranks as
    the bench reduces them -- first as computed, then with a mistake planted
    in rank 1's digests."""
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import ctypes
    from types import SimpleNamespace

    import torch
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from curtree_b200 import _lib
        from oracle import oracle as O
        L = _lib.load()
        boxes, windows = bench.make_query_inputs(rank, 30_000, 400)
        f = 16
        rsz = L.crt_tree_size(boxes.n, f)
        lv = (ctypes.c_int64 * 40)()
        nl = L.crt_tree_levels(boxes.n, f, lv, 40)
        sb, tr = O.build(boxes, f)
        sizes_ok = tr.sz == rsz and sum(lv[:nl]) == rsz and list(lv[:nl]) == O.levels(boxes.n, f)

        class Tree:
            def to_host(self):
                return tr

        class Sorted:
            def to_host(self):
                return sb

        st = O.tree_query_stats(tr, sb, windows)
        args = SimpleNamespace(fanout=f, parity_windows=0)
        flags = []
        for planted in (False, True):
            h = st.hashes.copy()
            if planted and rank == 1:
                h[123] ^= np.uint64(1)
            par = bench.parity_headline(args, boxes, windows, Tree(), Sorted(),
                                        {"persistent": (st.counts, h, 0)}, world)
            ok = torch.tensor([1 if par["ok"] else 0], dtype=torch.int32)
            dist.all_reduce(ok, op=dist.ReduceOp.MIN)
            flags.append((bool(par["ok"]), bool(ok.item()), par["windows_checked"]))
        out.put((rank, sizes_ok, int(st.counts.sum()), flags, _digest(sb)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_cpu_ranks_check_parity_of_their_own_batches():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_parity_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, n0, f0, t0), (r1, s1, n1, f1, t1) = res
    assert s0 and s1                          # library sizing = oracle sizing
    assert t0 == t1                           # the same replica tree on both ranks
    assert n0 > 0 and n1 > 0 and n0 != n1     # each rank its own batch
    assert f0[0] == (True, True, 400) and f1[0] == (True, True, 400)
    # the mistake on rank 1 fails its own check, and the reduced flag everywhere
    assert f0[1] == (True, False, 400) and f1[1] == (False, False, 400)


def test_single_process_reduce_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.5, None) == 3.5
