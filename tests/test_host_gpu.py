"""nspb_spgemm_host: operands and result in host memory, copies overlapped
with the row-blocked numeric phase; results against the oracle."""
import numpy as np
import pytest
import torch

import nsp_b200 as nb
import oracle
from nsp_b200._lib import ERR_CAPACITY
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def check(res, A, B, exact=True):
    rp, col, val = oracle.spgemm(A, B)
    assert_same_structure(np.asarray(res[0]), np.asarray(res[1]), rp, col)
    if exact:
        assert_bitwise(np.asarray(res[2]), val)
    else:
        assert_close(np.asarray(res[2]), val, oracle.absbound(A, B, rp, col))


class Pinned:
    def __init__(self, M):
        self.nrows, self.ncols = M.nrows, M.ncols
        self.rowptr = torch.from_numpy(M.rowptr).pin_memory()
        self.col = torch.from_numpy(M.col).pin_memory()
        self.val = torch.from_numpy(M.val).pin_memory()


@pytest.mark.parametrize("nblocks", [0, 1, 3, 64])
def test_host_product_blocks(cuda, nblocks):
    A = nb.gen.random(5000, 4000, 0, 30, seed=3)
    B = nb.gen.random(4000, 3500, 0, 12, seed=4)
    check(nb.spgemm_host(A, B, nblocks=nblocks), A, B)


def test_host_pinned_and_aliased(cuda):
    A = nb.gen.stencil(20, npts=27)
    pA = Pinned(A)
    n = A.nrows
    _, st = nb.spgemm(A.to_device(), A.to_device(), return_stats=True)
    out = (torch.empty(n + 1, dtype=torch.int32).pin_memory(),
           torch.empty(st["nnz"], dtype=torch.int32).pin_memory(),
           torch.empty(st["nnz"], dtype=torch.float64).pin_memory())
    res = nb.spgemm_host(pA, pA, out=out, nblocks=5)  # B's arrays are A's: copied once
    check(tuple(x.numpy() for x in res), A, A)


def test_host_long_rows_and_unsorted(cuda):
    P = nb.gen.powerlaw(30_000, max_deg=6000, seed=5)
    check(nb.spgemm_host(P, P, nblocks=7), P, P, exact=False)
    rng = np.random.default_rng(2)
    col = P.col.copy()
    for i in range(0, P.nrows, 4):
        rng.shuffle(col[P.rowptr[i]:P.rowptr[i + 1]])
    Pu = HostCSR(P.nrows, P.ncols, P.rowptr, col, P.val)
    check(nb.spgemm_host(P, Pu, nblocks=4), P, Pu, exact=False)


@pytest.mark.parametrize("nblocks", [2, 8, 40])
def test_host_banded_value_chunks(cuda, nblocks):
    # a banded A (rows reach only nearby B rows) with a separate B: row blocks
    # wait for the value chunks of their own rows; empty row ranges in A give
    # chunks without any column
    A = nb.gen.stencil_slab(24, 24, 24, 0, 24, npts=7)
    rp = A.rowptr.copy()
    lo, hi = 3000, 7000  # rows [lo, hi) emptied
    drop = rp[hi] - rp[lo]
    keep = np.r_[0:rp[lo], rp[hi]:A.nnz]
    rp[lo:hi + 1] = rp[lo]
    rp[hi + 1:] -= drop
    Ae = HostCSR(A.nrows, A.ncols, rp, A.col[keep], A.val[keep])
    B = nb.gen.stencil(24, npts=27)
    check(nb.spgemm_host(Ae, B, nblocks=nblocks), Ae, B, exact=True)
    check(nb.spgemm_host(Pinned(B), Pinned(B), nblocks=nblocks), B, B, exact=True)


def test_host_compensated_fp32(cuda):
    # fp32 host operands in the compensated mode: each row block's numeric step
    # takes its bins from the host row pointer in this mode too
    P = nb.gen.powerlaw(20_000, max_deg=2000, seed=12, fp32=True)  # fp32-representable
    P32 = HostCSR(P.nrows, P.ncols, P.rowptr, P.col, P.val.astype(np.float32))
    res = nb.spgemm_host(P32, P32, nblocks=6, precision="fp32c")
    rp, col, val = oracle.spgemm(P, P)
    assert_same_structure(np.asarray(res[0]), np.asarray(res[1]), rp, col)
    assert_close(np.asarray(res[2]), val, oracle.absbound(P, P, rp, col), tol=1e-10)


def test_host_capacity(cuda):
    A = nb.gen.random(300, 200, 1, 8, seed=6)
    B = nb.gen.random(200, 100, 1, 8, seed=7)
    rp = np.empty(301, np.int32)
    small = (rp, np.empty(5, np.int32), np.empty(5, np.float64))
    with pytest.raises(nb.NspbError) as e:
        nb.spgemm_host(A, B, out=small)
    assert e.value.status == ERR_CAPACITY
    want, _, _ = oracle.spgemm(A, B)
    assert np.array_equal(rp, want)  # the row pointer is written even then
