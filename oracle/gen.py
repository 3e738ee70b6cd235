"""TEST INFRASTRUCTURE — numpy restatement of the seeded stencil generator.

The benchmark's CPU reference arm builds its input here, so that arm loads no
part of the product library. Tests check it bit for bit against the
library's own generator (nspb_gen_stencil). It follows the same definition:
every off-diagonal value of the 27-point stencil is one draw of a
counter-based SplitMix64 mixer keyed by (seed, stream 27, lower row id,
higher row id), mapped to uniform[-1, 1); the diagonal is the sum of the
row's off-diagonal magnitudes, added in (dz, dy, dx) loop order, plus one.
The 7-point stencil has diagonal 6 and off-diagonals -1. Columns are
ascending within each row. The reference itself has no generator: it reads
matrices from files (src/READ_MATRIX_MPI.cpp:146-356).
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

_MASK = 0xFFFFFFFFFFFFFFFF


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _draw(seed: int, stream: int, row: np.ndarray, slot: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        s = np.uint64((seed ^ ((stream * 0x632BE59BD9B4E019) & _MASK)) & _MASK)
        base = _mix64(np.asarray(s, dtype=np.uint64))
        return _mix64(_mix64(base + row.astype(np.uint64)) + slot.astype(np.uint64))


def _unit_pm1(r: np.ndarray) -> np.ndarray:
    return 2.0 * ((r >> np.uint64(11)).astype(np.float64) * 2.0 ** -53) - 1.0


def stencil(L: int, npts: int = 27, seed: int = 20261203, fp32: bool = False):
    """The L^3 stencil as a SimpleNamespace(nrows, ncols, rowptr, col, val)."""
    assert npts in (7, 27)
    n = L * L * L
    i = np.arange(n, dtype=np.int64)
    x, y, z = i % L, (i // L) % L, i // (L * L)
    offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
            if npts == 27 or (dx != 0) + (dy != 0) + (dz != 0) <= 1]
    valid = np.stack([(x + dx >= 0) & (x + dx < L) & (y + dy >= 0) & (y + dy < L)
                      & (z + dz >= 0) & (z + dz < L) for dz, dy, dx in offs], axis=1)
    cols = np.stack([i + dx + L * dy + L * L * dz for dz, dy, dx in offs], axis=1)
    vals = np.zeros(cols.shape, dtype=np.float64)
    asum = np.zeros(n, dtype=np.float64)
    for q, (dz, dy, dx) in enumerate(offs):
        if (dz, dy, dx) == (0, 0, 0):
            continue
        if npts == 7:
            v = np.full(n, -1.0)
        else:
            j = np.where(valid[:, q], cols[:, q], i)
            v = _unit_pm1(_draw(seed, 27, np.minimum(i, j), np.maximum(i, j)))
            if fp32:
                v = v.astype(np.float32).astype(np.float64)
        v = np.where(valid[:, q], v, 0.0)
        vals[:, q] = v
        asum = asum + np.abs(v)  # the generator's loop order; 0.0 for absent entries
    d = offs.index((0, 0, 0))
    diag = np.full(n, 6.0) if npts == 7 else asum + 1.0
    if fp32 and npts == 27:
        diag = diag.astype(np.float32).astype(np.float64)
    vals[:, d] = diag
    counts = valid.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(counts, out=rowptr[1:])
    return SimpleNamespace(nrows=n, ncols=n, rowptr=rowptr,
                           col=cols[valid].astype(np.int32), val=vals[valid])
