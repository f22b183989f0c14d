"""Seeded synthetic sparse symmetric tensors (unique sorted index tuples).

The reference ships one input (examples/contact-5.tns); every other workload
is generated here from a seed so that the same tensor is produced on any
machine (numpy's PCG64 stream).  Tuples are returned 1-based and sorted
ascending within each tuple, as the reference loader leaves them
(src/utils/loader.cpp:29-31), and unique across the tensor.

Workloads (sizes are the ones the benchmark and tests use):
  * zipf_tuples        ids ~ Zipf(s) over a seeded rank->id permutation,
                       repeats inside a tuple allowed
  * planted_partition  a fraction of tuples drawn inside one of k equal
                       communities, the rest uniform over all ids
  * powerlaw_communities  Chung-Lu style weights w_i ~ i^(-1/(gamma-1)),
                       a fraction of tuples inside one community
"""
from __future__ import annotations

import os
import struct

import numpy as np

__all__ = [
    "zipf_tuples", "planted_partition", "powerlaw_communities", "uniform_values",
    "write_spt", "read_spt", "write_tns", "read_tns", "workload",
]


def _unique_rows(t: np.ndarray) -> np.ndarray:
    """Unique rows of a sorted-within-row uint32 matrix, first occurrence kept,
    original order preserved.  Each row is packed into as few 63-bit keys as
    hold it (most significant first), the rows are ordered by stable
    multi-threaded sorts of those keys, least significant key first, and the
    first row of every run of equal keys is kept."""
    import torch
    if t.shape[0] == 0:
        return t
    k, order = t.shape
    bits = max(1, int(t.max()).bit_length())
    per = 63 // bits
    keys = []
    for s0 in range(0, order, per):
        w = np.zeros(k, dtype=np.int64)
        for j in range(s0, min(order, s0 + per)):
            w = (w << bits) | t[:, j].astype(np.int64)
        keys.append(torch.from_numpy(w))
    perm = torch.arange(k)
    for w in reversed(keys):
        _, idx = torch.sort(w[perm], stable=True)
        perm = perm[idx]
    new_run = torch.zeros(k - 1, dtype=torch.bool)
    for w in keys:
        ws = w[perm]
        new_run |= ws[1:] != ws[:-1]
    keep = torch.ones(k, dtype=torch.bool)
    keep[1:] = new_run
    first, _ = torch.sort(perm[keep])
    return t[first.numpy()]


def _inverse_cdf(cdf: np.ndarray, u: np.ndarray) -> np.ndarray:
    """np.searchsorted(cdf, u, side="right"), computed with torch's
    multi-threaded search (the same comparisons, so the same indices)."""
    import torch
    r = torch.searchsorted(torch.from_numpy(np.ascontiguousarray(cdf)),
                           torch.from_numpy(np.ascontiguousarray(u)).reshape(-1), right=True)
    return r.numpy().reshape(u.shape)


def _draw_unique(draw, nnz: int, order: int, rng) -> np.ndarray:
    """Call draw(k) -> (k, order) uint32 ids (0-based) until nnz unique sorted
    tuples exist; returns them 1-based in draw order."""
    have = np.zeros((0, order), dtype=np.uint32)
    want = nnz
    for _ in range(200):
        k = int(max(1024, (want - have.shape[0]) * 1.3))
        t = draw(k)
        t.sort(axis=1)
        have = _unique_rows(np.concatenate([have, t], axis=0))
        if have.shape[0] >= want:
            break
    if have.shape[0] < want:
        raise ValueError(f"could not draw {nnz} unique tuples (got {have.shape[0]})")
    return (have[:want] + 1).astype(np.uint32)


def zipf_tuples(order: int, n: int, nnz: int, s: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    perm = rng.permutation(n).astype(np.uint32)

    def draw(k):
        r = _inverse_cdf(cdf, rng.random((k, order)))
        return perm[np.minimum(r, n - 1)]

    return _draw_unique(draw, nnz, order, rng)


def planted_partition(order: int, n: int, nnz: int, communities: int,
                      frac_in: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    size = n // communities

    def draw(k):
        inside = rng.random(k) < frac_in
        c = rng.integers(0, communities, size=k)
        t = rng.integers(0, n, size=(k, order), dtype=np.int64)
        loc = rng.integers(0, size, size=(k, order), dtype=np.int64) + (c * size)[:, None]
        t[inside] = loc[inside]
        return t.astype(np.uint32)

    return _draw_unique(draw, nnz, order, rng)


def powerlaw_communities(order: int, n: int, nnz: int, gamma: float,
                         communities: int, frac_in: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = np.arange(1, n + 1, dtype=np.float64) ** (-1.0 / (gamma - 1.0))
    perm = rng.permutation(n)
    weight = np.empty(n)
    weight[perm] = w
    comm = np.arange(n) % communities
    global_cdf = np.cumsum(weight)
    global_cdf /= global_cdf[-1]
    members = [np.nonzero(comm == c)[0] for c in range(communities)]
    cdfs = []
    for mem in members:
        cw = np.cumsum(weight[mem])
        cdfs.append(cw / cw[-1])

    def draw(k):
        t = np.empty((k, order), dtype=np.int64)
        inside = rng.random(k) < frac_in
        u = rng.random((k, order))
        g = np.minimum(_inverse_cdf(global_cdf, u), n - 1)
        t[:] = g
        cs = rng.integers(0, communities, size=k)
        for c in range(communities):
            sel = inside & (cs == c)
            if not np.any(sel):
                continue
            idx = np.minimum(_inverse_cdf(cdfs[c], u[sel]),
                             len(members[c]) - 1)
            t[sel] = members[c][idx]
        return t.astype(np.uint32)

    return _draw_unique(draw, nnz, order, rng)


def community_zipf(order: int, n: int, nnz: int, communities: int, s: float, seed: int,
                   frac_in: float = 0.9) -> np.ndarray:
    """Planted communities with Zipf(s) degrees inside each community: a
    fraction frac_in of the tuples draw all ids from one community (ranked by
    a seeded permutation), the rest draw ids Zipf(s) over all nodes."""
    rng = np.random.default_rng(seed)
    comm = rng.integers(0, communities, size=n)
    members = [np.nonzero(comm == c)[0] for c in range(communities)]
    members = [m if len(m) else np.array([c % n]) for c, m in enumerate(members)]
    cdfs = []
    for mem in members:
        w = np.arange(1, len(mem) + 1, dtype=np.float64) ** (-s)
        c = np.cumsum(w)
        cdfs.append(c / c[-1])
        rng.shuffle(mem)
    wall = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    call = np.cumsum(wall)
    call /= call[-1]
    perm = rng.permutation(n)

    def draw(k):
        t = perm[np.minimum(_inverse_cdf(call, rng.random((k, order))), n - 1)].astype(np.int64)
        inside = rng.random(k) < frac_in
        cs = rng.integers(0, communities, size=k)
        for c in range(communities):
            sel = inside & (cs == c)
            cnt = int(sel.sum())
            if not cnt:
                continue
            idx = np.minimum(_inverse_cdf(cdfs[c], rng.random((cnt, order))),
                             len(members[c]) - 1)
            t[sel] = members[c][idx]
        return t.astype(np.uint32)

    return _draw_unique(draw, nnz, order, rng)


def uniform_values(nnz: int, seed: int) -> np.ndarray:
    """values uniform in (0, 1], rounded to float32 and widened (exact in FP64)."""
    rng = np.random.default_rng(seed + 7919)
    v = 1.0 - rng.random(nnz)
    return v.astype(np.float32).astype(np.float64)


def workload(name: str, scale: float = 1.0, seed: int | None = None):
    """(order, dim, inds (nnz x order uint32 1-based), vals float64) for a named
    workload.  scale < 1 shrinks nnz (and n for the large ones) proportionally
    for bounded samples."""
    if name == "hooi_order5_zipf":          # order 5, n=250, 10k tuples, Zipf(1.2)
        order, n, nnz = 5, 250, int(10_000 * scale)
        t = zipf_tuples(order, n, nnz, 1.2, 0 if seed is None else seed)
        v = np.ones(nnz)
    elif name == "s3ttmc_order4_zipf":      # order 4, n=100k, 5M tuples, Zipf(1.1)
        order, n, nnz = 4, 100_000, int(5_000_000 * scale)
        t = zipf_tuples(order, n, nnz, 1.1, 1 if seed is None else seed)
        v = uniform_values(nnz, 1 if seed is None else seed)
    elif name == "mixed_order6_planted":    # order 6, n=50k, 2M tuples, 8 communities
        order, n, nnz = 6, 50_000, int(2_000_000 * scale)
        t = planted_partition(order, n, nnz, 8, 0.8, 2 if seed is None else seed)
        v = np.ones(nnz)
    elif name == "learned_order5_powerlaw":  # order 5, n=200k, 20M tuples
        order, n, nnz = 5, max(1000, int(200_000 * scale)), int(20_000_000 * scale)
        t = powerlaw_communities(order, n, nnz, 2.1, 16, 0.8, 4 if seed is None else seed)
        v = np.ones(nnz)
    else:
        raise KeyError(name)
    return order, n, t, v


# ------------------------------------------------------------------ file io

def write_spt(path: str, order: int, dim: int, inds: np.ndarray, vals: np.ndarray) -> None:
    """Binary tuple file: b'SPT1', u32 order, u32 dim, u32 0, u64 nnz,
    nnz*order u32 ids (1-based, sorted), nnz f64 values."""
    inds = np.ascontiguousarray(inds, dtype=np.uint32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    with open(path, "wb") as f:
        f.write(b"SPT1")
        f.write(struct.pack("<IIIQ", order, dim, 0, vals.shape[0]))
        f.write(inds.tobytes())
        f.write(vals.tobytes())


def read_spt(path: str):
    with open(path, "rb") as f:
        if f.read(4) != b"SPT1":
            raise ValueError("not an SPT1 file")
        order, dim, _, nnz = struct.unpack("<IIIQ", f.read(20))
        inds = np.frombuffer(f.read(4 * order * nnz), dtype=np.uint32).reshape(nnz, order)
        vals = np.frombuffer(f.read(8 * nnz), dtype=np.float64)
    return order, dim, inds.copy(), vals.copy()


def write_tns(path: str, order: int, dim: int, inds: np.ndarray, vals: np.ndarray) -> None:
    """Text .tns as read by the reference loader: 'order dim' then one
    'i1 ... iN value' line per nonzero."""
    with open(path, "w") as f:
        f.write(f"{order} {dim}\n")
        body = np.concatenate([inds.astype(np.float64), vals[:, None]], axis=1)
        fmt = " ".join(["%d"] * order) + " %.17g"
        np.savetxt(f, body, fmt=fmt)


def read_tns(path: str):
    with open(path) as f:
        head = f.readline().split()
        order, dim = int(head[0]), int(head[1])
        data = np.loadtxt(f, ndmin=2) if os.path.getsize(path) > 0 else np.zeros((0, order + 1))
    inds = np.sort(data[:, :order].astype(np.uint32), axis=1)
    return order, dim, inds, data[:, order].astype(np.float64)
