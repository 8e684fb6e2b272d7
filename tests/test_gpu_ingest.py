"""GPU ingest of the reference's MBR text format: crt_read_mbr_csv_device and
crt_parse_mbr_csv_device against the host loader crt_read_mbr_csv (itself
pinned to the reference's readMBR, src/utility.cpp:5-40, in test_io.py) and,
where the reference's CPU build is present, against readMBR directly.
Boxes and ids must be bit-identical, statuses and record counts equal."""
import ctypes
import decimal
import os
import tempfile

import numpy as np
import pytest

from curtree_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def crt():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import curtree_b200 as C
    C._lib.load()
    return C


def host_read(path, n, r):
    """The host loader: (status, n_read, [xmin, ymin, xmax, ymax], id)."""
    L = _lib.load()
    a = [np.zeros(max(n, 0), np.float32) for _ in range(4)]
    ids = np.zeros(max(n, 0), np.int32)
    got = ctypes.c_int64(0)
    st = L.crt_read_mbr_csv(str(path).encode(), n, r, *[x.ctypes.data for x in a], ids.ctypes.data,
                            ctypes.byref(got))
    return st, got.value, a, ids


def device_read(path, n, r):
    """crt_read_mbr_csv_device: (status, n_read, arrays, id) with the arrays
    copied back and the device box set freed."""
    import torch
    L = _lib.load()
    box = _lib.crt_bbox_f32()
    got = ctypes.c_int64(0)
    st = L.crt_read_mbr_csv_device(str(path).encode(), n, r, ctypes.byref(box), ctypes.byref(got),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if st != _lib.CRT_OK:
        assert not box.xmin and box.sz == 0, "nothing is handed out on an error"
        return st, got.value, None, None
    from curtree_b200.rtree import _d2h
    arrs = [_d2h(p, box.sz, np.float32) for p in (box.xmin, box.ymin, box.xmax, box.ymax)]
    ids = _d2h(box.id, box.sz, np.int32)
    assert L.crt_bbox_free(ctypes.byref(box)) == 0
    return st, got.value, arrs, ids


def device_parse(text: bytes, n, r):
    """crt_parse_mbr_csv_device on text in host memory into torch arrays."""
    import torch
    L = _lib.load()
    out = [torch.full((max(n, 1),), 7.0, dtype=torch.float32, device="cuda") for _ in range(4)]
    ids = torch.full((max(n, 1),), 7, dtype=torch.int32, device="cuda")
    buf = ctypes.create_string_buffer(text, len(text))
    got = ctypes.c_int64(0)
    st = L.crt_parse_mbr_csv_device(buf, len(text), n, r, *[t.data_ptr() for t in out],
                                    ids.data_ptr(), ctypes.byref(got),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st, got.value, [t.cpu().numpy()[:n] for t in out], ids.cpu().numpy()[:n]


def same(host, dev, text=""):
    hs, hn, ha, hi = host
    ds, dn, da, di = dev
    assert (ds, dn) == (hs, hn), (text[:300], host[:2], dev[:2])
    if hs == _lib.CRT_OK:
        for x, y in zip(ha, da):
            assert np.array_equal(x[:hn].view(np.uint32), y[:hn].view(np.uint32)), text[:300]
        assert np.array_equal(hi[:hn], di[:hn])


def check_text(tmp, text: str, n, r=0.0):
    path = os.path.join(tmp, "t.csv")
    raw = text.encode("latin-1")
    with open(path, "wb") as f:
        f.write(raw)
    host = host_read(path, n, r)
    same(host, device_parse(raw, n, r), text)
    return host


# ---- number spellings --------------------------------------------------------

def midpoint_strings(rng, k):
    """Decimal spellings of points halfway between two adjacent floats, exact
    and nudged by one unit in the 25th digit either way."""
    out = []
    ctx = decimal.Context(prec=60)
    short = decimal.Context(prec=28)
    for _ in range(k):
        a = np.float32(rng.uniform(1e-3, 1e6)) * np.float32(rng.choice([1, -1]))
        b = np.nextafter(a, np.float32(np.inf), dtype=np.float32)
        mid = ctx.divide(ctx.add(decimal.Decimal(float(a)), decimal.Decimal(float(b))), 2)
        s = format(mid, "f")
        out.append(s)
        nudge = ctx.scaleb(decimal.Decimal(1), mid.adjusted() - 24)
        out.append(format(short.add(mid, nudge), "e"))
        out.append(format(short.subtract(mid, nudge), "e"))
    return out


def number_pool(rng):
    pool = [f"{x:.6f}" for x in rng.uniform(-1e5, 1e5, 200)]
    pool += [repr(float(x)) for x in rng.uniform(-1e3, 1e3, 200)]
    pool += [f"{x:.{int(p)}e}" for x, p in zip(rng.uniform(-1, 1, 200) * 10.0 ** rng.integers(-45, 40, 200),
                                                  rng.integers(0, 20, 200))]
    pool += [float(x).hex() for x in rng.uniform(-10, 10, 20)]
    pool += ["inf", "-inf", "nan", "INFINITY", "NaN", "+inf", "-nan"]
    pool += midpoint_strings(rng, 60)
    pool += ["16777217", "16777219", "33554435", "-0", "+0", "-0.0", "+.5", "5.", "1E+05", "1e-05",
             "0" * 40 + "1.5", "1" + "0" * 30, "0." + "0" * 30 + "17", "123456789012345678901234567",
             "1.00000000000000000000000000001", "3.4028235e38", "3.4028236e38", "1e39", "-1e39",
             "1.17549435e-38", "1e-40", "1.4e-45", "7e-46", "2.5e-45", "0e99999", "1e-99999",
             "9" * 19, "9" * 20, "18446744073709551615", "0.1", "0.2", "0.3", "1e22", "1e23",
             "1.e3", "00000.0000", "4.9406564584124654e-324"]
    return pool


def int_pool(rng):
    ids = [str(x) for x in rng.integers(-2**31, 2**31 - 1, 200)]
    ids += ["0", "-0", "+7", "2147483647", "-2147483648", "2147483648", "4294967297",
            "-4294967297", "123456789012345678", "1234567890123456789", "99999999999999999999",
            "-99999999999999999999", "0000000000000000000000000042"]
    return ids


def test_number_spellings_match_host_loader(crt):
    rng = np.random.default_rng(3)
    nums, ints = number_pool(rng), int_pool(rng)
    lines = []
    for i in range(6000):
        f = [nums[j] for j in rng.integers(0, len(nums), 4)]
        k = [ints[j] for j in rng.integers(0, len(ints), 3)]
        lines.append(",".join(f + k))
    with tempfile.TemporaryDirectory() as tmp:
        for r in (0.0, 0.37):
            host = check_text(tmp, "\n".join(lines) + "\n", len(lines), r)
            assert host[0] == _lib.CRT_OK and host[1] == len(lines)


# ---- layout: blanks, line ends, lengths, malformed records ---------------------

LAYOUT_CASES = [
    "",
    "\n\n   \n\t\r\n",
    "1,2,3,4,5,6,7",
    "1,2,3,4,5,6,7\n",
    "1,2,3,4,5,6,7\r\n8,9,10,11,12,13,14\r\n",
    "  1, 2,\t3,\r4, 5, 6, 7  \n",
    "1,2,3,4,5,6,7 \t \n",
    "1,2,3,4,5,6,7,8,9,junk\n",
    "1,2,3,4,5,6,7\x00junk\n",
    "1,2,3,4,5,6,7\n\n\n  \n1,2,3,4,5,6,7\n",
    "\n\n1,2,3,4,5,6,7",
    "1,2,3 ,4,5,6,7\n",
    "1,2,3,4,5 ,6,7\n",
    "1,2,3,4\n",
    "1,2,3,4,5,6\n",
    "1,,3,4,5,6,7\n",
    ",1,2,3,4,5,6,7\n",
    "1,2,\n3,4,5,6,7\n",
    "1,2,3,4,5,6,\n7\n",
    "x,2,3,4,5,6,7\n",
    "1,2,3,4,5.5,6,7\n",
    "1,2,3,4,5,6,7x\n",
    "1,2,3,4,5,6,7\n1,2,3,4,5,6\n",
    "\v1,2,3,4,5,6,7\n",
    "1,\v2,3,4,5,6,7\n",
    "1,\f2,3,4,5,6,7\n",
    "1," + " " * 100 + "2,3,4,5,6,7\n",
    "1e5,2E-3,3,4,5,6,7\n",
    "1e,2,3,4,5,6,7\n",
    "1e+,2,3,4,5,6,7\n",
    "0x1p3,2,3,4,5,6,7\n",
    "1," + "1" * 61 + ",3,4,5,6,7\n",
    "1," + "1" * 62 + ",3,4,5,6,7\n",
    "1," + "1" * 63 + ",3,4,5,6,7\n",
    "1," + "1" * 64 + ",3,4,5,6,7\n",
    "1,2,3,4,5,6," + "7" * 70 + "\n",
    "1,2,3,4,5,6," + "7" * 62 + "\n",
    "1,2,3,4,5,6,7" + " " * 70 + "\n",
    "1,2,3,4," + "1" * 70 + ",6,7\n",
    "-,2,3,4,5,6,7\n",
    ".,2,3,4,5,6,7\n",
    "+-1,2,3,4,5,6,7\n",
    "1..2,2,3,4,5,6,7\n",
    "1,2,3,4,-,6,7\n",
    "\r\r\r1,2,3,4,5,6,7\r\r\n",
    # fscanf's records are not the lines: across lines, several on a line,
    # whatever follows the seventh number starting the next record
    "1,2,\n3,4,5,6,7\n8,9,10,11,12,13,14\n",
    "1,2,3,4,5,6,7 8,9,10,11,12,13,14\n",
    "1,2,3,4,5,6,7\t\v\f8,9,10,11,12,13,14",
    "1,2,3,4,5,6,7,8\n9,9,9,9,9,9,9\n",
    "1,2,3,4,5,6,7x\n8,9,10,11,12,13,14\n",
    "1,2,3,4,5,6,7-8,9,10,11,12,13,14\n",
    "1,\n2,\n3,\n4,\n5,\n6,\n7\n",
    "1.5e3,2,3,4,5,6,7 8,9,10,11,12,13,14 15,16,17,18,19,20,21",
    "1,2,3,4\n,5,6,7\n",
    "1,2,3,4,5,6,7\r8,9,10,11,12,13,14\n",
]


@pytest.mark.parametrize("case", range(len(LAYOUT_CASES)))
def test_layout_cases_match_host_loader(crt, case):
    text = LAYOUT_CASES[case]
    with tempfile.TemporaryDirectory() as tmp:
        for n in (0, 1, 2, 3):
            check_text(tmp, text, n, 0.5)


def test_first_malformed_record_is_reported(crt):
    rng = np.random.default_rng(9)
    good = [f"{a:.5f},{b:.5f},{a + 1:.5f},{b + 1:.5f},{i},0,0" for i, (a, b) in
            enumerate(rng.uniform(0, 100, (40000, 2)))]
    with tempfile.TemporaryDirectory() as tmp:
        for bad_at in (0, 1, 17_000, 39_999):
            lines = list(good)
            lines[bad_at] = lines[bad_at].replace(",", " ,", 1)
            if bad_at + 5 < len(lines):
                lines[bad_at + 5] = "junk"
            host = check_text(tmp, "\n".join(lines) + "\n", len(lines))
            assert host[0] == _lib.CRT_ERR_INVALID_ARG and host[1] == bad_at


# ---- whole files: formats, sizes, counts -----------------------------------------

def make_rows(n, seed):
    rng = np.random.default_rng(seed)
    x1 = rng.uniform(-1e5, 1e5, n)
    y1 = rng.uniform(-1e5, 1e5, n)
    x2 = x1 + rng.normal(0, 50, n)
    y2 = y1 + rng.normal(0, 50, n)
    ids = rng.integers(-2**31, 2**31 - 1, n)
    return list(zip(x1, y1, x2, y2, ids, rng.integers(0, 100, n), rng.integers(0, 9, n)))


FORMATS = {
    "plain": lambda r: f"{r[0]:.6f},{r[1]:.6f},{r[2]:.6f},{r[3]:.6f},{r[4]},{r[5]},{r[6]}",
    "long": lambda r: f"{float(r[0])!r},{float(r[1])!r},{float(r[2])!r},{float(r[3])!r},{r[4]},{r[5]},{r[6]}",
    "sci": lambda r: f"{r[0]:.9e},{r[1]:.3e},{r[2]:.12e},{r[3]:g},{r[4]},{r[5]},{r[6]}",
    "spaced": lambda r: f" {r[0]:.4f}, {r[1]:.4f},\t{r[2]:.4f},{r[3]:.4f}, {r[4]},{r[5]},{r[6]}  ",
}


@pytest.mark.parametrize("fmt", sorted(FORMATS))
def test_formats_match_host_loader_and_reference(crt, fmt):
    rows = make_rows(300_000, seed=len(fmt))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "mbr.csv")
        with open(path, "w") as f:
            f.write("\n".join(FORMATS[fmt](r) for r in rows) + "\n")
        for r in (0.0, 10.0):
            host = host_read(path, len(rows), r)
            assert host[0] == _lib.CRT_OK
            same(host, device_read(path, len(rows), r))
            same(host, device_read(path, -1, r))
        if O.ref_cpu_available():
            ref = O.ref_read_mbr(path, len(rows), 0.0)
            st, got, a, ids = device_read(path, len(rows), 0.0)
            for mine, theirs in zip(a, (ref.xmin, ref.ymin, ref.xmax, ref.ymax)):
                assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32))
            assert np.array_equal(ids, ref.id)


def test_large_file_counts_and_prefixes(crt):
    rows = make_rows(1_500_000, seed=77)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "big.csv")
        with open(path, "w") as f:
            f.write("\r\n".join(FORMATS["plain"](r) for r in rows))
        n = len(rows)
        host = host_read(path, n, 0.25)
        same(host, device_read(path, n, 0.25))
        same(host_read(path, 1_000_003, 0.25), device_read(path, 1_000_003, 0.25))
        st, got, _, _ = device_read(path, n + 1, 0.25)
        assert (st, got) == (_lib.CRT_ERR_INVALID_ARG, n)
        st, got, a, _ = device_read(path, 0, 0.25)
        assert (st, got, len(a[0])) == (_lib.CRT_OK, 0, 0)


def test_many_host_parsed_records(crt):
    """More undecided records (hex spellings) than the device's first list
    holds: the parse runs again into a list of their exact count, host
    threads finish them, and the result is the host loader's."""
    rng = np.random.default_rng(5)
    n = (1 << 20) + 5000
    xs = rng.uniform(-10, 10, (n, 4))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "hex.csv")
        with open(path, "w") as f:
            f.write("\n".join(f"{float(a).hex()},{b:.3f},{c:.3f},{d:.3f},{i},1,2"
                              for i, (a, b, c, d) in enumerate(xs)) + "\n")
        host = host_read(path, n, 1.0)
        assert host[0] == _lib.CRT_OK
        same(host, device_read(path, n, 1.0))
        lines = open(path).read().split("\n")
        lines[n - 3] = "1,2,3 ,4,5,6,7"
        with open(path, "w") as f:
            f.write("\n".join(lines))
        host = host_read(path, n, 1.0)
        assert host[:2] == (_lib.CRT_ERR_INVALID_ARG, n - 3)
        same(host, device_read(path, n, 1.0))


def test_python_reader_and_build(crt):
    rows = make_rows(50_000, seed=4)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "p.csv")
        with open(path, "w") as f:
            f.write("\n".join(FORMATS["long"](r) for r in rows) + "\n")
        b = crt.read_mbr_csv(path, r=2.0)
        host = host_read(path, len(rows), 2.0)
        assert b.sz == len(rows)
        hb = b.to_host()
        for x, y in zip(host[2], (hb.xmin, hb.ymin, hb.xmax, hb.ymax)):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        assert np.array_equal(host[3], hb.id)
        rt = crt.RTree(10)
        crt.build_rtree(b, rt)
        assert rt.sz == crt.tree_size(len(rows), 10)
        with pytest.raises(crt.CrtError):
            crt.read_mbr_csv(path, n=len(rows) + 1)
        with pytest.raises(crt.CrtError):
            crt.read_mbr_csv(os.path.join(tmp, "missing.csv"))


# ---- binary records ---------------------------------------------------------------

def bin_read(path, n, r):
    import torch
    L = _lib.load()
    box = _lib.crt_bbox_f32()
    got = ctypes.c_int64(0)
    st = L.crt_read_mbr_bin_device(str(path).encode(), n, r, ctypes.byref(box), ctypes.byref(got),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if st != _lib.CRT_OK:
        assert not box.xmin and box.sz == 0
        return st, got.value, None, None
    from curtree_b200.rtree import _d2h
    arrs = [_d2h(p, box.sz, np.float32) for p in (box.xmin, box.ymin, box.xmax, box.ymax)]
    ids = _d2h(box.id, box.sz, np.int32)
    assert L.crt_bbox_free(ctypes.byref(box)) == 0
    return st, got.value, arrs, ids


def expected_boxes(rec, r):
    """readMBR's box of each binary record, in fp32 (std::min / std::max
    keep the first endpoint unless the second compares below / above it).
    numpy computes on the host, like readMBR, so a NaN corner keeps its sign
    and payload here; the device must do the same."""
    r = np.float32(r)
    x1, y1, x2, y2 = (rec[k] for k in ("x1", "y1", "x2", "y2"))
    return [np.where(x2 < x1, x2, x1) - r, np.where(y2 < y1, y2, y1) - r,
            np.where(x1 < x2, x2, x1) + r, np.where(y1 < y2, y2, y1) + r]


def test_binary_records_match_readmbr_arithmetic(crt):
    from curtree_b200 import datasets as D
    rng = np.random.default_rng(12)
    n = 700_001
    rec = np.empty(n, D.MBR_BIN_RECORD)
    for k in ("x1", "y1", "x2", "y2"):
        rec[k] = rng.uniform(-1e5, 1e5, n).astype(np.float32)
    special = np.array([np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-45, -3.4e38], np.float32)
    for k in ("x1", "y1", "x2", "y2"):
        idx = rng.integers(0, n, 2000)
        rec[k][idx] = special[rng.integers(0, len(special), 2000)]
    rec["id"] = rng.integers(-2**31, 2**31 - 1, n)
    rec["pid"], rec["nume"] = 1, 2
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "m.bin")
        rec.tofile(path)
        for r in (0.0, 0.37):
            st, got, a, ids = bin_read(path, -1, r)
            assert (st, got) == (_lib.CRT_OK, n)
            for mine, want in zip(a, expected_boxes(rec, r)):
                assert np.array_equal(mine.view(np.uint32), want.view(np.uint32))
            assert np.array_equal(ids, rec["id"])
        st, got, a, ids = bin_read(path, 1000, 1.0)
        assert (st, got, len(ids)) == (_lib.CRT_OK, 1000, 1000)
        assert np.array_equal(ids, rec["id"][:1000])
        assert bin_read(path, n + 1, 0.0)[:2] == (_lib.CRT_ERR_INVALID_ARG, n)
        with open(path, "ab") as f:
            f.write(b"\0" * 5)
        assert bin_read(path, -1, 0.0)[0] == _lib.CRT_ERR_INVALID_ARG
        open(path, "wb").close()
        st, got, a, ids = bin_read(path, -1, 0.0)
        assert (st, got, len(ids)) == (_lib.CRT_OK, 0, 0)


def test_binary_and_text_forms_agree(crt):
    """The same boxes written as text (nine significant digits: exact in
    fp32) and as binary records load to identical device boxes."""
    from curtree_b200 import datasets as D
    b = D.uniform_boxes(200_000, seed=31)
    b.id[:] = np.random.default_rng(32).integers(-2**31, 2**31 - 1, b.n)
    raw = D.mbr_bin_bytes(b, seed=5)
    rec = np.frombuffer(raw, D.MBR_BIN_RECORD)
    with tempfile.TemporaryDirectory() as tmp:
        pb, pt = os.path.join(tmp, "m.bin"), os.path.join(tmp, "m.csv")
        with open(pb, "wb") as f:
            f.write(raw)
        with open(pt, "w") as f:
            f.write("".join(f"{x1:.9g},{y1:.9g},{x2:.9g},{y2:.9g},{i},{p},{q}\n"
                            for x1, y1, x2, y2, i, p, q in rec.tolist()))
        same(device_read(pt, b.n, 0.5), bin_read(pb, b.n, 0.5))
        x = crt.read_mbr_bin(pb, r=0.5).to_host()
        y = crt.read_mbr_csv(pt, r=0.5).to_host()
        for u, v in zip((x.xmin, x.ymin, x.xmax, x.ymax), (y.xmin, y.ymin, y.xmax, y.ymax)):
            assert np.array_equal(u.view(np.uint32), v.view(np.uint32))
        assert np.array_equal(x.id, b.id) and np.array_equal(y.id, b.id)


def test_read_all_records_as_fscanf_finds_them(crt):
    """n = -1 (every record of the file): where fscanf's records are not the
    lines, the device loader returns the host loader's records all the same,
    and as many of them."""
    texts = [c for c in LAYOUT_CASES if c.count(",") >= 6]
    with tempfile.TemporaryDirectory() as tmp:
        for text in texts:
            path = os.path.join(tmp, "t.csv")
            with open(path, "wb") as f:
                f.write(text.encode("latin-1"))
            hs, hn, ha, hi = host_read(path, 64, 0.5)  # 64 > any record count here
            ds, dn, da, di = device_read(path, -1, 0.5)
            if ds == _lib.CRT_OK:
                assert dn == hn, text
                for x, y in zip(ha, da):
                    assert np.array_equal(x[:hn].view(np.uint32), y.view(np.uint32)), text
                assert np.array_equal(hi[:hn], di), text
            else:
                assert ds == _lib.CRT_ERR_INVALID_ARG and dn == hn, (text, hs, hn, ds, dn)
