"""Ingest without a GPU: crt_read_mbr_csv (host code in the library) against
the reference's own readMBR compiled from src/utility.cpp -- bit-identical
boxes and ids -- and its error statuses where the reference exits or throws."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from curtree_b200 import _lib
from oracle import oracle as O


def write_csv(path, rows, fmt):
    with open(path, "w") as f:
        for r in rows:
            f.write(fmt(r) + "\n")


def read_ours(path, n, r):
    L = _lib.load()
    a = [np.empty(n, np.float32) for _ in range(4)]
    ids = np.empty(n, np.int32)
    got = ctypes.c_int64(0)
    st = L.crt_read_mbr_csv(path.encode(), n, r, *[x.ctypes.data for x in a], ids.ctypes.data,
                            ctypes.byref(got))
    return st, got.value, a, ids


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


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
@pytest.mark.parametrize("fmt", sorted(FORMATS))
@pytest.mark.parametrize("r", [0.0, 10.0, 0.37])
def test_read_mbr_matches_reference(fmt, r):
    rows = make_rows(5000, seed=hash(fmt) % 1000)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "mbr.csv")
        write_csv(path, rows, FORMATS[fmt])
        ref = O.ref_read_mbr(path, len(rows), r)
        st, got, a, ids = read_ours(path, len(rows), r)
        assert st == _lib.CRT_OK and got == len(rows)
        for mine, theirs in zip(a, (ref.xmin, ref.ymin, ref.xmax, ref.ymax)):
            assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32))
        assert np.array_equal(ids, ref.id)


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
def test_blank_before_separator_rejected_like_reference():
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "b.csv")
        with open(path, "w") as f:
            f.write("1,2,3,4,5,6,7\n1,2,3 ,4,5,6,7\n")
        with pytest.raises(ValueError):
            O.ref_read_mbr(path, 2, 0.0)
        st, got, _, _ = read_ours(path, 2, 0.0)
        assert st == _lib.CRT_ERR_INVALID_ARG and got == 1


def test_read_mbr_errors():
    with tempfile.TemporaryDirectory() as tmp:
        st, got, _, _ = read_ours(os.path.join(tmp, "missing.csv"), 10, 0.0)
        assert st == _lib.CRT_ERR_INVALID_ARG
        path = os.path.join(tmp, "short.csv")
        write_csv(path, make_rows(7, 1), FORMATS["plain"])
        st, got, _, _ = read_ours(path, 10, 0.0)
        assert st == _lib.CRT_ERR_INVALID_ARG and got == 7
        path = os.path.join(tmp, "bad.csv")
        with open(path, "w") as f:
            f.write("1,2,3,4,5,6,7\n1,2,x,4,5,6,7\n1,2,3,4,5,6,7\n")
        st, got, _, _ = read_ours(path, 3, 0.0)
        assert st == _lib.CRT_ERR_INVALID_ARG and got == 1
        assert b"record 1" in _lib.load().crt_last_error()


def test_device_reader_argument_errors_need_no_gpu():
    """crt_read_mbr_csv_device / crt_parse_mbr_csv_device reject bad
    arguments, a missing file and a directory before touching a device."""
    L = _lib.load()
    box = _lib.crt_bbox_f32()
    got = ctypes.c_int64(5)
    with tempfile.TemporaryDirectory() as tmp:
        for path, n in ((None, 1), (os.path.join(tmp, "missing.csv").encode(), 1), (tmp.encode(), 1),
                        (os.path.join(tmp, "x.csv").encode(), -2)):
            st = L.crt_read_mbr_csv_device(path, n, 0.0, ctypes.byref(box), ctypes.byref(got), None)
            assert st == _lib.CRT_ERR_INVALID_ARG and got.value in (0, 5)
            assert not box.xmin and box.sz == 0
    assert L.crt_parse_mbr_csv_device(None, 10, 1, 0.0, None, None, None, None, None,
                                      ctypes.byref(got), None) == _lib.CRT_ERR_INVALID_ARG
    assert L.crt_parse_mbr_csv_device(b"1,2,3,4,5,6,7\n", 14, 1, 0.0, None, None, None, None, None,
                                      ctypes.byref(got), None) == _lib.CRT_ERR_INVALID_ARG


def test_mbr_text_generator_matches_python_formatting():
    """datasets.mbr_csv_text writes what Python's %.6f / %d would, and the
    host loader reads it back to the same boxes."""
    from curtree_b200 import datasets as D
    rng = np.random.default_rng(8)
    n = 3000
    b = D.HostBoxes(*(rng.uniform(-4e4, 4e4, n).astype(np.float32) for _ in range(4)),
                    rng.integers(-2**31, 2**31 - 1, n).astype(np.int32))
    b.xmin[:3] = [0.0, -0.0000004, 123456.5]
    b.id[:2] = [-2**31, 2**31 - 1]
    text = D.mbr_csv_text(b, seed=9)
    g = np.random.default_rng(9)
    swap = g.random(n) < 0.5
    pid, nume = g.integers(0, 100, n), g.integers(0, 10, n)
    want = []
    for i in range(n):
        x1, y1, x2, y2 = ((b.xmax[i], b.ymax[i], b.xmin[i], b.ymin[i]) if swap[i]
                          else (b.xmin[i], b.ymin[i], b.xmax[i], b.ymax[i]))
        want.append(f"{x1:.6f},{y1:.6f},{x2:.6f},{y2:.6f},{b.id[i]},{pid[i]},{nume[i]}\n")
    assert text.decode() == "".join(want)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "g.csv")
        with open(path, "wb") as f:
            f.write(text)
        st, got, a, ids = read_ours(path, n, 0.0)
        assert st == _lib.CRT_OK and got == n and np.array_equal(ids, b.id)
        lo = np.minimum(b.xmin, b.xmax)
        assert np.allclose(a[0], lo, rtol=0, atol=1e-2)


def test_binary_reader_size_errors_need_no_gpu():
    """crt_read_mbr_bin_device checks the file's size against whole 28-byte
    records and against n before touching a device."""
    L = _lib.load()
    box = _lib.crt_bbox_f32()
    got = ctypes.c_int64(0)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "m.bin")
        with open(path, "wb") as f:
            f.write(b"\0" * (28 * 3 + 1))
        assert L.crt_read_mbr_bin_device(path.encode(), -1, 0.0, ctypes.byref(box),
                                         ctypes.byref(got), None) == _lib.CRT_ERR_INVALID_ARG
        with open(path, "wb") as f:
            f.write(b"\0" * (28 * 3))
        assert L.crt_read_mbr_bin_device(path.encode(), 4, 0.0, ctypes.byref(box),
                                         ctypes.byref(got), None) == _lib.CRT_ERR_INVALID_ARG
        assert got.value == 3 and not box.xmin
        assert L.crt_read_mbr_bin_device(os.path.join(tmp, "none").encode(), 1, 0.0,
                                         ctypes.byref(box), ctypes.byref(got),
                                         None) == _lib.CRT_ERR_INVALID_ARG


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
def test_multi_chunk_file_matches_reference():
    """A file large enough for the record-start scan to split across host
    threads (8 MiB chunks), with blank lines, CRLF ends, indented records and
    a blank stretch longer than a chunk, reads like the reference's readMBR."""
    rng = np.random.default_rng(17)
    rows = make_rows(400_000, seed=18)
    seps = ["\n", "\r\n", "\n\n", "\n   \n", "\n\t \r\n", "\n  "]
    parts = []
    for i, r in enumerate(rows):
        parts.append(FORMATS["plain"](r))
        parts.append(seps[rng.integers(0, len(seps))])
        if i == 150_000:
            parts.append(" \t\r\n" * (3 << 20))  # 12 MiB without a record
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "big.csv")
        with open(path, "w") as f:
            f.write("".join(parts))
        assert os.path.getsize(path) > 3 * (8 << 20)
        for n in (len(rows), 150_002, 1):
            ref = O.ref_read_mbr(path, n, 0.5)
            st, got, a, ids = read_ours(path, n, 0.5)
            assert st == _lib.CRT_OK and got == n
            for mine, theirs in zip(a, (ref.xmin, ref.ymin, ref.xmax, ref.ymax)):
                assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32))
            assert np.array_equal(ids, ref.id)
        st, got, _, _ = read_ours(path, len(rows) + 1, 0.5)
        assert (st, got) == (_lib.CRT_ERR_INVALID_ARG, len(rows))


# Texts where fscanf's records are not the lines: readMBR reads each record
# with fscanf(fp, "%f,%f,%f,%f,%d,%d,%d\n", ...), whose numbers skip any
# whitespace before them (newlines too) and whose closing "\n" skips any
# whitespace after the last one -- so a record may span lines, several may
# share a line, and what follows the seventh number starts the next record.
FSCANF_TEXTS = [
    ("1,2,\n3,4,5,6,7\n8,9,10,11,12,13,14\n", 2),
    ("1,2,3,4,5,6,7 8,9,10,11,12,13,14\n", 2),
    ("1,2,3,4,5,6,7\t\v\f8,9,10,11,12,13,14", 2),
    ("1,2,3,4,5,6,7,8\n9,9,9,9,9,9,9\n", 2),
    ("1,2,3,4,5,6,7x\n8,9,10,11,12,13,14\n", 2),
    ("1,2,3,4,5,6,7-8,9,10,11,12,13,14\n", 2),
    ("\n\n  1,2,3,4,5,6,7\n\n\n8,9,10,11,12,13,14\n\n", 2),
    ("1,\n2,\n3,\n4,\n5,\n6,\n7\n", 1),
    ("1.5e3,2,3,4,5,6,7 8,9,10,11,12,13,14 15,16,17,18,19,20,21", 3),
    ("1,2,3,4,5,6,7\n", 2),
    ("1,2,3,4\n,5,6,7\n", 1),
]


def ref_records(path, n):
    """How many records the reference's readMBR reads before it throws (it
    throws at the first record fscanf cannot read, end of file included)."""
    for k in range(n, 0, -1):
        try:
            O.ref_read_mbr(path, k, 0.0)
            return k
        except ValueError:
            continue
    return 0


@pytest.mark.skipif(not O.ref_cpu_available(), reason="reference CPU build absent")
@pytest.mark.parametrize("text,n", FSCANF_TEXTS)
def test_records_found_as_fscanf_finds_them(text, n):
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "t.csv")
        with open(path, "w") as f:
            f.write(text)
        k = ref_records(path, n)
        st, got, a, ids = read_ours(path, n, 0.25)
        assert got == k
        assert (st == _lib.CRT_OK) == (k == n)
        if k == n:
            ref = O.ref_read_mbr(path, n, 0.25)
            for mine, theirs in zip(a, (ref.xmin, ref.ymin, ref.xmax, ref.ymax)):
                assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32))
            assert np.array_equal(ids, ref.id)
