"""Seeded CSR generators (host), thin wrappers of the library's
nspb_gen_* functions. Every value depends only on (seed, row, slot)."""
from __future__ import annotations

import numpy as np

from ._lib import check, lib
from .csr import HostCSR

DEFAULT_SEED = 20261203


def _two_call(nrows, fn, *args, fp32=False):
    rowptr = np.empty(nrows + 1, dtype=np.int32)
    nnz = fn(*args, int(fp32), rowptr.ctypes.data, None, None)
    if nnz < 0:
        check(int(nnz), fn.__name__)
    col = np.empty(nnz, dtype=np.int32)
    val = np.empty(nnz, dtype=np.float64)
    got = fn(*args, int(fp32), rowptr.ctypes.data, col.ctypes.data, val.ctypes.data)
    if got < 0:
        check(int(got), fn.__name__)
    return rowptr, col, val


def stencil(nx: int, ny: int | None = None, nz: int | None = None, npts: int = 27,
            seed: int = DEFAULT_SEED, fp32: bool = False) -> HostCSR:
    """3-D 7-point (diag 6, off -1) or 27-point (symmetric off-diagonal
    uniform[-1,1], diag = sum|off| + 1) stencil on nx*ny*nz, columns sorted."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    n = nx * ny * nz
    rp, col, val = _two_call(n, lib.nspb_gen_stencil, nx, ny, nz, npts, seed, fp32=fp32)
    return HostCSR(n, n, rp, col, val)


def powerlaw(nrows: int = 1_000_000, ncols: int | None = None, alpha: float = 2.1,
             mean_deg: float = 16.0, max_deg: int = 50_000, seed: int = DEFAULT_SEED,
             fp32: bool = False) -> HostCSR:
    """Rows with truncated-Pareto degrees (mean `mean_deg`, cap `max_deg`),
    columns uniform without duplicates, values uniform[-1,1]."""
    ncols = nrows if ncols is None else ncols
    rp, col, val = _two_call(nrows, lib.nspb_gen_powerlaw, nrows, ncols, alpha, mean_deg,
                             max_deg, seed, fp32=fp32)
    return HostCSR(nrows, ncols, rp, col, val)


def random(nrows: int, ncols: int, dmin: int, dmax: int, seed: int = DEFAULT_SEED,
           fp32: bool = False) -> HostCSR:
    """Rows with degree uniform in [dmin, dmax], columns uniform without
    duplicates, values uniform[-1,1]."""
    rp, col, val = _two_call(nrows, lib.nspb_gen_random, nrows, ncols, dmin, dmax, seed,
                             fp32=fp32)
    return HostCSR(nrows, ncols, rp, col, val)


def powerlaw_xmin(alpha=2.1, mean_deg=16.0, max_deg=50_000) -> float:
    return float(lib.nspb_powerlaw_xmin(alpha, mean_deg, max_deg))


def stencil_slab(nx: int, ny: int, nz: int, z0: int, z1: int, npts: int = 27,
                 seed: int = DEFAULT_SEED, fp32: bool = False) -> HostCSR:
    """Rows of z-planes [z0, z1) of the nx*ny*nz stencil, global column ids."""
    n = nx * ny * (z1 - z0)
    rp, col, val = _two_call(n, lib.nspb_gen_stencil_slab, nx, ny, nz, z0, z1, npts, seed,
                             fp32=fp32)
    return HostCSR(n, nx * ny * nz, rp, col, val)
