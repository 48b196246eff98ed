"""Compact digests of a product C, shared by the fixture generator and the tests.

A digest pins a result matrix too large to store whole:

  * ``samples``: C at ``count`` positions drawn from a counter-based stream
    (the splitmix64 generator of oracle.uniform, so positions are identical on
    every machine and numpy version).  A quarter of the rows are drawn from
    the rows that dynamic peeling computes (the fringe left by the floor
    sub-blocking at every recursion level, linalg/linalg.hpp:201-244), a
    quarter of the columns likewise, the rest uniformly;
  * ``rowsum`` / ``colsum``: sums of C over ``groups`` equal bands of rows
    (all columns) and of columns (all rows), a checksum of every entry.

Values are stored as base64 of little-endian float64 bytes.
"""

from __future__ import annotations

import base64

import numpy as np

_GOLD = np.uint64(0x9E3779B97F4A7C15)


def _stream(count: int, seed: int, stream: int) -> np.ndarray:
    """count uint64 values of the splitmix64 stream (seed, stream)."""
    with np.errstate(over="ignore"):
        key = np.uint64(seed) * np.uint64(0xD1B54A32D192ED03) + np.uint64(stream) * np.uint64(0x8CB92BA72F3D8DD7)
        e = np.arange(1, count + 1, dtype=np.uint64)
        z = key + e * _GOLD
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def fringe(size: int, base: int, steps: int) -> list:
    """Indices along one dimension (``size``, split ``base`` ways per level,
    ``steps`` levels) that fall in a peeled fringe at some level."""
    out = []

    def walk(off, length, level):
        if level == steps or base <= 1:
            return
        blk = length // base
        core = blk * base
        out.extend(range(off + core, off + length))
        if blk == 0:
            return
        for i in range(base):
            walk(off + i * blk, blk, level + 1)

    walk(0, size, 0)
    return sorted(set(out))


def positions(m: int, n: int, m0: int, n0: int, steps: int, count: int, seed: int):
    """(rows, cols) int64 arrays of ``count`` sample positions."""
    z = _stream(4 * count, seed, 77)
    r = (z[:count] % np.uint64(max(m, 1))).astype(np.int64)
    c = (z[count:2 * count] % np.uint64(max(n, 1))).astype(np.int64)
    fr = np.array(fringe(m, m0, steps), dtype=np.int64)
    fc = np.array(fringe(n, n0, steps), dtype=np.int64)
    q = count // 4
    if fr.size:
        r[:q] = fr[(z[2 * count:2 * count + q] % np.uint64(fr.size)).astype(np.int64)]
    if fc.size:
        c[q:2 * q] = fc[(z[3 * count:3 * count + q] % np.uint64(fc.size)).astype(np.int64)]
    return r, c


def bands(size: int, groups: int):
    g = max(1, min(size, groups))
    return [(i * size // g, (i + 1) * size // g) for i in range(g)]


def digest_np(C: np.ndarray, rows, cols, groups: int) -> dict:
    """Digest of a numpy matrix (any order)."""
    m, n = C.shape
    samples = C[rows, cols].astype(np.float64)
    col_tot = C.sum(axis=0)
    row_tot = C.sum(axis=1)
    rowsum = np.array([row_tot[a:b].sum() for a, b in bands(m, groups)])
    colsum = np.array([col_tot[a:b].sum() for a, b in bands(n, groups)])
    return {"samples": samples, "rowsum": rowsum, "colsum": colsum}


def digest_torch(C, rows, cols, groups: int) -> dict:
    """The same digest of a (CUDA) torch matrix, returned as numpy arrays."""
    import torch

    m, n = C.shape
    ri = torch.as_tensor(rows, device=C.device)
    ci = torch.as_tensor(cols, device=C.device)
    samples = C[ri, ci].double().cpu().numpy()
    col_tot = C.double().sum(dim=0)
    row_tot = C.double().sum(dim=1)
    rowsum = torch.stack([row_tot[a:b].sum() for a, b in bands(m, groups)]).cpu().numpy()
    colsum = torch.stack([col_tot[a:b].sum() for a, b in bands(n, groups)]).cpu().numpy()
    return {"samples": samples, "rowsum": rowsum, "colsum": colsum}


def enc(a: np.ndarray) -> str:
    return base64.b64encode(np.ascontiguousarray(a, dtype="<f8").tobytes()).decode()


def dec(s: str) -> np.ndarray:
    return np.frombuffer(base64.b64decode(s), dtype="<f8").copy()


def rel_diffs(want: dict, got: dict) -> dict:
    """max |got - want| / |want| per digest part (NaN terms skipped, as in
    MaxRelativeDiff, linalg/linalg.hpp:280-295)."""
    out = {}
    for key in ("samples", "rowsum", "colsum"):
        w = np.asarray(want[key], dtype=np.float64)
        g = np.asarray(got[key], dtype=np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = np.abs(g - w) / np.abs(w)
        r = r[~np.isnan(r)]
        out[key] = float(r.max()) if r.size else 0.0
    out["max"] = max(out.values())
    return out
