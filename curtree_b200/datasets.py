"""Seeded synthetic box and window sets for the R-tree workloads.

Every generator draws in the unit square [0, 1)^2 and then multiplies each
coordinate by 2**15.  The factor is a power of two, so the scaling is exact in
fp32: every `<`/`>` comparison, and so every hit pair, is the same as on the
unscaled data.  It also turns the reference's truncating `(ushort)` cast of the
box centre (src/rtree_bulkload_thrust.cuh:55-56) into a 15-bit-per-axis
quantisation, i.e. a 30-bit Morton key; on raw [0, 1) data every key would be 0.

Box ids are positional (`id = index`), matching how the reference's drivers
verify (src/rtree_test_frontier.cu:102-123).

Workloads (sizes are the defaults; every function takes `n`/`nq` so the tests
can use small instances of the same distributions):
  uniform_boxes        1M boxes, centres U[0,1)^2, width/height U[0, 1e-3]
  uniform_windows      10k windows, centres U[0,1)^2, side U[0, 1e-2]
  clustered_boxes      100M boxes: 1000 Gaussian clusters (sigma log-U[1e-4,1e-2])
                       + 10% uniform, side log-normal(ln 1e-4, 1), 1% exact
                       duplicates, 1% zero-area boxes
  mixed_windows        1M windows, side log-U[1e-5, 1e-1], centres half uniform,
                       half drawn from the box centres
  road_boxes           50M boxes on 100 random segments, Pareto(1.5) sides in
                       [1e-6, 0.5], aspect ratio up to 1e4
  road_windows         2M windows: 50% points, 40% small, 10% covering >1% of
                       the domain
"""
from __future__ import annotations

import dataclasses

import numpy as np

SCALE = np.float32(2.0 ** 15)


@dataclasses.dataclass
class HostBoxes:
    """Host-side box set in the reference's BBOX<float> layout (src/rtree.h:3-11):
    four fp32 coordinate arrays and an int32 id array, structure of arrays."""

    xmin: np.ndarray
    ymin: np.ndarray
    xmax: np.ndarray
    ymax: np.ndarray
    id: np.ndarray

    @property
    def n(self) -> int:
        return int(self.xmin.shape[0])

    def take(self, idx) -> "HostBoxes":
        return HostBoxes(self.xmin[idx], self.ymin[idx], self.xmax[idx], self.ymax[idx], self.id[idx])

    def slice(self, a: int, b: int) -> "HostBoxes":
        return HostBoxes(self.xmin[a:b], self.ymin[a:b], self.xmax[a:b], self.ymax[a:b], self.id[a:b])

    def copy(self) -> "HostBoxes":
        return HostBoxes(self.xmin.copy(), self.ymin.copy(), self.xmax.copy(), self.ymax.copy(),
                         self.id.copy())

    @staticmethod
    def concat(parts) -> "HostBoxes":
        parts = list(parts)
        return HostBoxes(*(np.concatenate([getattr(p, f) for p in parts])
                           for f in ("xmin", "ymin", "xmax", "ymax", "id")))

    def write_crtb(self, path: str) -> None:
        """Write the CRTB box file the reference runners read: magic, int64 n,
        then xmin, ymin, xmax, ymax (fp32) and id (int32)."""
        with open(path, "wb") as f:
            f.write(b"CRTB")
            f.write(np.int64(self.n).tobytes())
            for a in (self.xmin, self.ymin, self.xmax, self.ymax):
                f.write(np.ascontiguousarray(a, dtype=np.float32).tobytes())
            f.write(np.ascontiguousarray(self.id, dtype=np.int32).tobytes())


def _boxes(cx, cy, w, h, scale=True) -> HostBoxes:
    """Boxes [c - w/2, c + w/2] rounded once to fp32, then scaled by 2^15."""
    cx = np.asarray(cx, np.float64)
    cy = np.asarray(cy, np.float64)
    hw = 0.5 * np.asarray(w, np.float64)
    hh = 0.5 * np.asarray(h, np.float64)
    xmin = (cx - hw).astype(np.float32)
    xmax = (cx + hw).astype(np.float32)
    ymin = (cy - hh).astype(np.float32)
    ymax = (cy + hh).astype(np.float32)
    if scale:
        xmin *= SCALE
        xmax *= SCALE
        ymin *= SCALE
        ymax *= SCALE
    ids = np.arange(xmin.shape[0], dtype=np.int32)
    return HostBoxes(xmin, ymin, xmax, ymax, ids)


def _unit_points(rng, n):
    return rng.random(n), rng.random(n)


def uniform_boxes(n: int = 1_000_000, seed: int = 1, max_side: float = 1e-3,
                  scale: bool = True) -> HostBoxes:
    """Centres uniform in [0,1)^2, width and height independently U[0, max_side]."""
    rng = np.random.default_rng(seed)
    cx, cy = _unit_points(rng, n)
    w = rng.random(n) * max_side
    h = rng.random(n) * max_side
    return _boxes(cx, cy, w, h, scale)


def uniform_windows(nq: int = 10_000, seed: int = 101, max_side: float = 1e-2,
                    scale: bool = True) -> HostBoxes:
    """Square windows, centres uniform in [0,1)^2, side U[0, max_side]."""
    rng = np.random.default_rng(seed)
    cx, cy = _unit_points(rng, nq)
    s = rng.random(nq) * max_side
    return _boxes(cx, cy, s, s, scale)


def clustered_boxes(n: int = 100_000_000, seed: int = 2, chunk: int = 10_000_000) -> HostBoxes:
    """Centres from 1000 isotropic Gaussians (sigma log-uniform in [1e-4, 1e-2])
    plus 10% uniform background, rejected into [0,1)^2; width and height
    log-normal(mu = ln 1e-4, sigma = 1); 1% of the boxes are exact duplicates of
    other boxes and 1% are zero-area points.  Generated in fixed-size chunks so
    the result does not depend on the host's memory."""
    ss = np.random.SeedSequence(seed)
    rng0 = np.random.default_rng(ss.spawn(1)[0])
    mu = rng0.random((1000, 2))
    sig = np.exp(rng0.uniform(np.log(1e-4), np.log(1e-2), 1000))
    parts = []
    for ci, cs in enumerate(ss.spawn((n + chunk - 1) // chunk)):
        rng = np.random.default_rng(cs)
        m = min(chunk, n - ci * chunk)
        cx = np.empty(m)
        cy = np.empty(m)
        filled = 0
        while filled < m:
            r = m - filled
            bg = rng.random(r) < 0.10
            k = rng.integers(0, 1000, r)
            x = np.where(bg, rng.random(r), mu[k, 0] + sig[k] * rng.standard_normal(r))
            y = np.where(bg, rng.random(r), mu[k, 1] + sig[k] * rng.standard_normal(r))
            ok = (x >= 0) & (x < 1) & (y >= 0) & (y < 1)
            c = int(ok.sum())
            cx[filled:filled + c] = x[ok]
            cy[filled:filled + c] = y[ok]
            filled += c
        w = rng.lognormal(np.log(1e-4), 1.0, m)
        h = rng.lognormal(np.log(1e-4), 1.0, m)
        pts = rng.random(m) < 0.01
        w[pts] = 0.0
        h[pts] = 0.0
        b = _boxes(cx, cy, w, h)
        dup = np.nonzero(rng.random(m) < 0.01)[0]
        if dup.size:
            src = rng.integers(0, m, dup.size)
            for f in ("xmin", "ymin", "xmax", "ymax"):
                a = getattr(b, f)
                a[dup] = a[src]
        parts.append(b)
    out = HostBoxes.concat(parts)
    out.id = np.arange(out.n, dtype=np.int32)
    return out


def mixed_windows(nq: int = 1_000_000, boxes: HostBoxes | None = None, seed: int = 103,
                  lo: float = 1e-5, hi: float = 1e-1) -> HostBoxes:
    """Square windows with side log-uniform in [lo, hi]; half the centres are
    uniform in [0,1)^2, half are the centres of randomly drawn boxes."""
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), nq))
    cx, cy = _unit_points(rng, nq)
    if boxes is not None and boxes.n:
        half = rng.random(nq) < 0.5
        pick = rng.integers(0, boxes.n, nq)
        bx = (boxes.xmin[pick].astype(np.float64) + boxes.xmax[pick]) / 2 / float(SCALE)
        by = (boxes.ymin[pick].astype(np.float64) + boxes.ymax[pick]) / 2 / float(SCALE)
        cx = np.where(half, bx, cx)
        cy = np.where(half, by, cy)
    return _boxes(cx, cy, s, s)


def road_boxes(n: int = 50_000_000, seed: int = 5, n_segments: int = 100,
               chunk: int = 10_000_000) -> HostBoxes:
    """Centres on `n_segments` random line segments (plus a 1e-4 jitter),
    rejected into [0,1)^2; long side Pareto(alpha = 1.5, min 1e-6) capped at
    0.5, short side = long / aspect with aspect log-uniform in [1, 1e4],
    oriented along x or y at random."""
    ss = np.random.SeedSequence(seed)
    rng0 = np.random.default_rng(ss.spawn(1)[0])
    p0 = rng0.random((n_segments, 2))
    p1 = rng0.random((n_segments, 2))
    parts = []
    for ci, cs in enumerate(ss.spawn((n + chunk - 1) // chunk)):
        rng = np.random.default_rng(cs)
        m = min(chunk, n - ci * chunk)
        cx = np.empty(m)
        cy = np.empty(m)
        filled = 0
        while filled < m:
            r = m - filled
            k = rng.integers(0, n_segments, r)
            t = rng.random(r)
            x = p0[k, 0] + t * (p1[k, 0] - p0[k, 0]) + 1e-4 * rng.standard_normal(r)
            y = p0[k, 1] + t * (p1[k, 1] - p0[k, 1]) + 1e-4 * rng.standard_normal(r)
            ok = (x >= 0) & (x < 1) & (y >= 0) & (y < 1)
            c = int(ok.sum())
            cx[filled:filled + c] = x[ok]
            cy[filled:filled + c] = y[ok]
            filled += c
        long_side = np.minimum(1e-6 * (1.0 + rng.pareto(1.5, m)), 0.5)
        aspect = np.exp(rng.uniform(0.0, np.log(1e4), m))
        short_side = long_side / aspect
        along_x = rng.random(m) < 0.5
        w = np.where(along_x, long_side, short_side)
        h = np.where(along_x, short_side, long_side)
        parts.append(_boxes(cx, cy, w, h))
    out = HostBoxes.concat(parts)
    out.id = np.arange(out.n, dtype=np.int32)
    return out


def road_windows(nq: int = 2_000_000, seed: int = 105) -> HostBoxes:
    """50% degenerate point windows, 40% small windows (side log-uniform in
    [1e-5, 1e-3]) and 10% windows covering more than 1% of the domain (side
    uniform in [0.1, 0.3])."""
    rng = np.random.default_rng(seed)
    cx, cy = _unit_points(rng, nq)
    u = rng.random(nq)
    small = np.exp(rng.uniform(np.log(1e-5), np.log(1e-3), nq))
    big = rng.uniform(0.1, 0.3, nq)
    s = np.where(u < 0.5, 0.0, np.where(u < 0.9, small, big))
    return _boxes(cx, cy, s, s)


def serving_requests(n_requests: int, n_trees: int, seed: int = 104,
                     lo: int = 1, hi: int = 100_000):
    """Request stream for the serving loop: tree index uniform over the trees,
    batch size log-uniform in [lo, hi] windows."""
    rng = np.random.default_rng(seed)
    tree = rng.integers(0, n_trees, n_requests)
    size = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), n_requests)).astype(np.int64)
    size = np.clip(size, lo, hi)
    return tree, size


def _digit_count(a: np.ndarray) -> np.ndarray:
    nd = np.ones(a.shape, np.int8)
    for k in range(1, 19):
        nd += a >= 10 ** k
    return nd


def mbr_csv_text(boxes: HostBoxes, decimals: int = 6, seed: int = 106) -> bytes:
    """The boxes as the reference's MBR text records "x1,y1,x2,y2,id,pid,nume",
    one per line (the format readMBR reads, src/utility.cpp:5-40): corners
    printed with `decimals` fraction digits, the corners of half of the
    records given in the opposite order (readMBR takes min/max of the
    endpoints), pid in [0, 100), nume in [0, 10).  Vectorised numpy: the
    records are laid out in a fixed-width byte matrix (numbers right-aligned,
    NUL padding) whose padding is then squeezed out."""
    rng = np.random.default_rng(seed)
    n = boxes.n
    swap = rng.random(n) < 0.5
    f64 = lambda a: np.asarray(a, np.float64)
    fields = [np.where(swap, f64(boxes.xmax), f64(boxes.xmin)),
              np.where(swap, f64(boxes.ymax), f64(boxes.ymin)),
              np.where(swap, f64(boxes.xmin), f64(boxes.xmax)),
              np.where(swap, f64(boxes.ymin), f64(boxes.ymax)),
              np.asarray(boxes.id, np.int64), rng.integers(0, 100, n), rng.integers(0, 10, n)]
    scale = 10 ** decimals
    parts = []  # (neg, integer part, its digit count, its widest count, fraction or None)
    for k, v in enumerate(fields):
        neg = v < 0
        if k < 4:
            q = np.rint(np.abs(v) * scale).astype(np.int64)
            ip, fp = q // scale, q % scale
        else:
            ip, fp = np.abs(v).astype(np.int64), None
        nd = _digit_count(ip)
        parts.append((neg, ip, nd, int(nd.max(initial=1)), fp))
    width = sum(1 + w + (1 + decimals if fp is not None else 0) + 1 for _, _, _, w, fp in parts)
    M = np.zeros((width, n), np.uint8)  # column-major while writing, rows at the end
    c = 0
    for k, (neg, ip, nd, w, fp) in enumerate(parts):
        # column c: room for the sign; digits right-aligned in c+1 .. c+w
        x = ip
        for j in range(w):
            x, d = np.divmod(x, 10)
            M[c + w - j] = np.where(nd > j, 48 + d, 0)
        M[c + w - nd[neg], np.flatnonzero(neg)] = ord("-")
        c += 1 + w
        if fp is not None:
            M[c] = ord(".")
            x = fp
            for j in range(decimals):
                x, d = np.divmod(x, 10)
                M[c + decimals - j] = 48 + d
            c += 1 + decimals
        M[c] = ord(",") if k < 6 else ord("\n")
        c += 1
    flat = np.ascontiguousarray(M.T).ravel()
    return flat[flat != 0].tobytes()


MBR_BIN_RECORD = np.dtype([("x1", "<f4"), ("y1", "<f4"), ("x2", "<f4"), ("y2", "<f4"),
                           ("id", "<i4"), ("pid", "<i4"), ("nume", "<i4")])


def mbr_bin_bytes(boxes: HostBoxes, seed: int = 106) -> bytes:
    """The boxes as 28-byte binary MBR records (float32 x1, y1, x2, y2, int32
    id, pid, nume, little-endian): the fields of mbr_csv_text with the same
    corner order and pid/nume draws, the corners kept exactly in fp32."""
    rng = np.random.default_rng(seed)
    n = boxes.n
    swap = rng.random(n) < 0.5
    rec = np.empty(n, MBR_BIN_RECORD)
    f32 = lambda a: np.asarray(a, np.float32)
    rec["x1"] = np.where(swap, f32(boxes.xmax), f32(boxes.xmin))
    rec["y1"] = np.where(swap, f32(boxes.ymax), f32(boxes.ymin))
    rec["x2"] = np.where(swap, f32(boxes.xmin), f32(boxes.xmax))
    rec["y2"] = np.where(swap, f32(boxes.ymin), f32(boxes.ymax))
    rec["id"] = boxes.id
    rec["pid"] = rng.integers(0, 100, n)
    rec["nume"] = rng.integers(0, 10, n)
    return rec.tobytes()
