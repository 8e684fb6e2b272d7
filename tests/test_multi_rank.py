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


def test_single_process_reduce_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.5, None) == 3.5
