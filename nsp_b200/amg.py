"""Smoothed-aggregation AMG Galerkin hierarchy and the batched workload.

The reference comes from an AMG solver whose setup forms the coarse
operators R·A·P with its SpGEMM (the Galerkin products the MPI product of
src/spspmpi.cu serves). This module builds that hierarchy on one GPU with
this library's product:

  level l: A_l (n_l x n_l), aggregates of 3x3x3 nodes (the last aggregate of
  a dimension is ragged when the edge is not a multiple of 3),
  P_tent(i, agg(i)) = 1, P = (I - w D^-1 A) P_tent with w = 2/3, R = P^T,
  A_{l+1} = R (A P).

Transposes and the smoothing update run on the host (setup code, not the
measured path); the products A·P_tent, A·P and R·(AP) run through nspb.
"""
from __future__ import annotations

import numpy as np

from .csr import HostCSR


def _transpose(M: HostCSR) -> HostCSR:
    """CSR transpose with columns ascending in every row (stable by row)."""
    rows = np.repeat(np.arange(M.nrows, dtype=np.int64), np.diff(M.rowptr))
    order = np.argsort(M.col, kind="stable")
    tcol = rows[order].astype(np.int32)
    tval = M.val[order]
    counts = np.bincount(M.col, minlength=M.ncols)
    trp = np.zeros(M.ncols + 1, dtype=np.int64)
    np.cumsum(counts, out=trp[1:])
    return HostCSR(M.ncols, M.nrows, trp.astype(np.int32), tcol, tval)


def _tentative(nx: int, ny: int, nz: int, agg: int = 3):
    """P_tent of the grid aggregation: node (x, y, z) -> (x//agg, y//agg, z//agg)."""
    cx, cy, cz = -(-nx // agg), -(-ny // agg), -(-nz // agg)
    idx = np.arange(nx * ny * nz, dtype=np.int64)
    x, y, z = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    coarse = (x // agg) + cx * ((y // agg) + cy * (z // agg))
    P = HostCSR(nx * ny * nz, cx * cy * cz, np.arange(nx * ny * nz + 1, dtype=np.int32),
                coarse.astype(np.int32), np.ones(nx * ny * nz))
    return P, (cx, cy, cz)


def _product(A: HostCSR, B: HostCSR) -> HostCSR:
    from . import spgemm
    return spgemm(A.to_device(), B.to_device()).to_host()


def smoothed_prolongator(A: HostCSR, Ptent: HostCSR, omega: float = 2.0 / 3.0) -> HostCSR:
    """P = P_tent - omega D^-1 (A P_tent). The pattern of A·P_tent contains
    agg(i) in row i (a_ii != 0), so P shares that pattern."""
    AP = _product(A, Ptent)
    rows = np.repeat(np.arange(A.nrows), np.diff(A.rowptr))
    diag = np.zeros(A.nrows)
    on = A.col == rows
    diag[rows[on]] = A.val[on]
    prow = np.repeat(np.arange(AP.nrows), np.diff(AP.rowptr))
    val = -omega * AP.val / diag[prow]
    tent = Ptent.col[prow] == AP.col
    val[tent] += 1.0
    return HostCSR(AP.nrows, AP.ncols, AP.rowptr, AP.col, val)


def hierarchy(A0: HostCSR, grid, levels: int = 4, omega: float = 2.0 / 3.0):
    """[(A_l, P_l, R_l, AP_l)] for l = 0 .. levels-2, and the coarsest A."""
    out = []
    A, (nx, ny, nz) = A0, grid
    for _ in range(levels - 1):
        Pt, (nx, ny, nz) = _tentative(nx, ny, nz)
        P = smoothed_prolongator(A, Pt, omega)
        R = _transpose(P)
        AP = _product(A, P)
        Ac = _product(R, AP)
        out.append((A, P, R, AP))
        A = Ac
    return out, A


def amg_batch(L: int = 96, levels: int = 4, seed: int = 20261203):
    """The 2*(levels-1) Galerkin products (A_l·P_l, R_l·(A_l P_l)) of the
    27-point stencil on L^3, as independent (A, B) pairs."""
    from .gen import stencil
    A0 = stencil(L, npts=27, seed=seed)
    levs, _ = hierarchy(A0, (L, L, L), levels)
    pairs = []
    for A, P, R, AP in levs:
        pairs.append((A, P))
        pairs.append((R, AP))
    return pairs


def random_batch(count: int = 256, nmin: int = 1000, nmax: int = 100_000, dmin: int = 4,
                 dmax: int = 32, seed: int = 20261203):
    """`count` independent random products A·B, n uniform in [nmin, nmax],
    degrees uniform in [dmin, dmax], columns uniform without duplicates."""
    from .gen import random
    rng = np.random.default_rng(seed)
    pairs = []
    for p in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        pairs.append((random(n, n, dmin, dmax, seed=seed + 2 * p),
                      random(n, n, dmin, dmax, seed=seed + 2 * p + 1)))
    return pairs
