"""Drop-in proof on the GPU: a C++ caller written like the reference's driver,
compiled against crtree/rtree_compat.h (once with crtree/rtree.h, once with
the reference's own rtree.h and utility.cuh), builds the tree and queries
through the C ABI; its node arrays and canonical pairs equal the oracle's."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from curtree_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVERS = [os.path.join(ROOT, "_build", n) for n in ("dropin_standalone", "dropin_refutil")]


def read_pairs(path):
    raw = np.fromfile(path, np.uint8)
    n = int(raw[:8].view(np.int64)[0])
    return raw[8:8 + 4 * n].view(np.int32), raw[8 + 4 * n:8 + 8 * n].view(np.int32)


@pytest.mark.parametrize("driver", DRIVERS, ids=[os.path.basename(d) for d in DRIVERS])
def test_dropin_driver(driver):
    if not os.path.exists(driver):
        if driver.endswith("refutil"):
            pytest.skip("reference-utility build needs the reference sources at build time")
        raise AssertionError(f"{driver} missing: run `make -C tests/cpp`")
    b = D.uniform_boxes(200_000, seed=60)
    q = D.mixed_windows(3000, b, seed=160, lo=1e-4, hi=2e-2)
    with tempfile.TemporaryDirectory() as tmp:
        bf, qf = os.path.join(tmp, "b.crtb"), os.path.join(tmp, "q.crtb")
        b.write_crtb(bf)
        q.write_crtb(qf)
        p = subprocess.run([driver, bf, qf, "10", os.path.join(tmp, "out")], capture_output=True,
                           text=True, timeout=300)
        assert p.returncode == 0, p.stdout + p.stderr
        sb, t = O.build(b, 10)
        raw = np.fromfile(os.path.join(tmp, "out_tree.bin"), np.uint8)
        rsz = int(raw[:8].view(np.int64)[0])
        assert rsz == t.sz
        body = raw[8:]
        for k, name in enumerate(("xmin", "ymin", "xmax", "ymax", "pos", "len")):
            got = body[4 * rsz * k:4 * rsz * (k + 1)].view(np.uint32)
            assert np.array_equal(got, getattr(t, name).view(np.uint32)), name
        want = O.canonical_pairs(*O.tree_query_pairs(t, sb, q))
        for form in ("frontier", "thrust"):
            fid, tid = read_pairs(os.path.join(tmp, f"out_{form}.bin"))
            assert np.array_equal(fid, want[0]) and np.array_equal(tid, want[1]), form
