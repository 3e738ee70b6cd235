"""Smoothed-aggregation AMG Galerkin hierarchy and the batched workload.

The reference comes from an AMG solver whose setup forms the coarse
operators R·A·P with its SpGEMM (the Galerkin products the MPI product of
src/spspmpi.cu serves). This module builds that hierarchy on one GPU with
this library's device entry points:

  level l: A_l (n_l x n_l), aggregates of 3x3x3 nodes (the last aggregate of
  a dimension is ragged when the edge is not a multiple of 3),
  P_tent(i, agg(i)) = 1                       (host: the aggregation map)
  P = (I - w D^-1 A) P_tent, w = 2/3          nspb_sa_prolongator
  R = P^T                                     nspb_transpose
  A_{l+1} = R (A P)                           two nspb_spgemm products
"""
from __future__ import annotations

import numpy as np

from .csr import HostCSR


def _tentative(nx: int, ny: int, nz: int, agg: int = 3):
    """P_tent of the grid aggregation: node (x, y, z) -> (x//agg, y//agg, z//agg)."""
    cx, cy, cz = -(-nx // agg), -(-ny // agg), -(-nz // agg)
    idx = np.arange(nx * ny * nz, dtype=np.int64)
    x, y, z = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    coarse = (x // agg) + cx * ((y // agg) + cy * (z // agg))
    P = HostCSR(nx * ny * nz, cx * cy * cz, np.arange(nx * ny * nz + 1, dtype=np.int32),
                coarse.astype(np.int32), np.ones(nx * ny * nz))
    return P, (cx, cy, cz)


def hierarchy(A0: HostCSR, grid, levels: int = 4, omega: float = 2.0 / 3.0):
    """[(A_l, P_l, R_l, AP_l)] for l = 0 .. levels-2 (host copies), and the
    coarsest A. Every operator is formed on the GPU."""
    from . import sa_prolongator, spgemm, transpose
    out = []
    nx, ny, nz = grid
    dA = A0.to_device()
    for _ in range(levels - 1):
        Pt, (nx, ny, nz) = _tentative(nx, ny, nz)
        dP = sa_prolongator(dA, Pt.to_device(), omega)
        dR = transpose(dP)
        dAP = spgemm(dA, dP)
        dAc = spgemm(dR, dAP)
        out.append((dA.to_host(), dP.to_host(), dR.to_host(), dAP.to_host()))
        dA = dAc
    return out, dA.to_host()


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
