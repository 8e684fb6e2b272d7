"""The autotuner: it times every candidate, returns the fastest, caches it,
and every candidate configuration answers with the same pairs."""
import os
import tempfile

import numpy as np
import pytest

from curtree_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_autotune_picks_and_caches():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    from curtree_b200.autotune import autotune, query_opts
    b = D.uniform_boxes(400_000, seed=97)
    q = D.mixed_windows(4000, b, seed=197)
    d = C.BBox.from_host(b)
    dq = C.BBox.from_host(q)
    with tempfile.TemporaryDirectory() as tmp:
        cache = os.path.join(tmp, "tune.json")
        best = autotune(d, dq, fanouts=(8, 16, 32), warps=(8, 32), stage=(0, 2, 3),
                        window_warps=(1, 2), chunks=(1024, 4096), reps=2, cache_path=cache)
        assert best["fanout"] in (8, 16, 32) and best["warps_per_cta"] in (8, 32)
        # every fanout x warps pair, then each other dimension's other values
        assert len(best["table"]) == 3 * 2 + 2 + 1 + 1
        assert {r["stage_levels"] for r in best["table"]} == {0, 2, 3}
        assert {r["warps_per_window"] for r in best["table"]} == {1, 2}
        assert best["ms"] == min(r["ms"] for r in best["table"])
        again = autotune(d, dq, cache_path=cache)
        assert again.get("cached") and again["fanout"] == best["fanout"]
    # the input was not reordered, and the chosen configuration is exact
    assert np.array_equal(d.id.cpu().numpy(), b.id)
    sorted_boxes, rt = C.build_into(d, best["fanout"])
    fid, tid = C.query(rt, sorted_boxes, dq, **query_opts(best))
    got = O.canonical_pairs(fid.cpu().numpy(), tid.cpu().numpy())
    sb, t = O.build(b, best["fanout"])
    want = O.canonical_pairs(*O.tree_query_pairs(t, sb, q))
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
