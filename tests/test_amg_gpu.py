"""AMG Galerkin driver on the GPU: CSR transpose (CSRm::T, src/CSR.cu:738-785),
the smoothed-aggregation prolongator (with CSRm::diag, src/CSR.cu:1389-1418)
and A_c = R (A P), against numpy restatements and the oracle."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200 import amg
from nsp_b200._lib import ERR_INVALID
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def np_transpose(M: HostCSR) -> HostCSR:
    """Stable transpose: within a column, entries keep their row-major order."""
    rows = np.repeat(np.arange(M.nrows, dtype=np.int64), np.diff(M.rowptr))
    order = np.argsort(M.col, kind="stable")
    trp = np.zeros(M.ncols + 1, dtype=np.int64)
    np.cumsum(np.bincount(M.col, minlength=M.ncols), out=trp[1:])
    return HostCSR(M.ncols, M.nrows, trp.astype(np.int32), rows[order].astype(np.int32),
                   M.val[order])


def np_sa_prolongator(A: HostCSR, Pt: HostCSR, omega: float) -> HostCSR:
    """(-omega * (A Pt)_ij) / a_ii, plus Pt_ij where Pt has an entry."""
    rp, col, val = oracle.spgemm(A, Pt)
    rows = np.repeat(np.arange(A.nrows), np.diff(A.rowptr))
    diag = np.zeros(A.nrows)
    on = A.col == rows
    diag[rows[on]] = A.val[on]  # the last diagonal entry of a row wins
    prow = np.repeat(np.arange(A.nrows), np.diff(rp))
    out = (-omega * val) / diag[prow]
    for i in range(Pt.nrows):
        for t in range(Pt.rowptr[i], Pt.rowptr[i + 1]):
            hit = rp[i] + np.searchsorted(col[rp[i]:rp[i + 1]], Pt.col[t])
            out[hit] += Pt.val[t]
    return HostCSR(A.nrows, Pt.ncols, rp, col, out)


def same(got: HostCSR, want: HostCSR):
    assert (got.nrows, got.ncols) == (want.nrows, want.ncols)
    assert_same_structure(got.rowptr, got.col, want.rowptr, want.col)
    assert_bitwise(got.val, want.val)


@pytest.mark.parametrize("shape", [(3000, 700, 0, 12), (500, 1, 0, 1), (200, 300_000, 1, 40)])
def test_transpose_matches_stable_restatement(cuda, shape):
    n, m, dmin, dmax = shape
    M = nb.gen.random(n, m, dmin, dmax, seed=n + m)
    same(nb.transpose(M.to_device()).to_host(), np_transpose(M))


def test_transpose_duplicates_fp32_and_empty(cuda):
    # duplicate (row, col) entries keep their stored order
    M = HostCSR(3, 4, np.array([0, 3, 3, 6], np.int32), np.array([2, 0, 2, 2, 3, 2], np.int32),
                np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0]))
    same(nb.transpose(M.to_device()).to_host(), np_transpose(M))
    F = nb.gen.random(400, 350, 0, 9, seed=2)
    dF = F.to_device()
    dF.val = dF.val.float()
    got = nb.transpose(dF)
    assert str(got.val.dtype) == "torch.float32"
    want = np_transpose(F)
    assert np.array_equal(got.col.cpu().numpy(), want.col)
    assert np.array_equal(got.val.cpu().numpy(), want.val.astype(np.float32))
    E = HostCSR(5, 7, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0))
    t = nb.transpose(E.to_device()).to_host()
    assert t.nrows == 7 and t.ncols == 5 and t.nnz == 0 and list(t.rowptr) == [0] * 8


def test_sa_prolongator_bitwise(cuda):
    A = nb.gen.stencil(12, npts=27)
    Pt, _ = amg._tentative(12, 12, 12)
    got = nb.sa_prolongator(A.to_device(), Pt.to_device(), 2.0 / 3.0).to_host()
    same(got, np_sa_prolongator(A, Pt, 2.0 / 3.0))


def test_sa_prolongator_missing_diagonal(cuda):
    A = nb.gen.random(50, 50, 1, 4, seed=3)
    keep = A.col != np.repeat(np.arange(50), np.diff(A.rowptr))
    rows = np.repeat(np.arange(50), np.diff(A.rowptr))[keep]
    rp = np.zeros(51, np.int32)
    np.cumsum(np.bincount(rows, minlength=50), out=rp[1:])
    A0 = HostCSR(50, 50, rp, A.col[keep], A.val[keep])  # no diagonal anywhere
    Pt, _ = amg._tentative(50, 1, 1)
    with pytest.raises(nb.NspbError) as e:
        nb.sa_prolongator(A0.to_device(), Pt.to_device())
    assert e.value.status == ERR_INVALID


def test_galerkin_matches_oracle(cuda):
    A = nb.gen.stencil(15, npts=27)
    Pt, _ = amg._tentative(15, 15, 15)
    P = np_sa_prolongator(A, Pt, 2.0 / 3.0)
    Ac, R = nb.galerkin(A.to_device(), P.to_device(), return_R=True)
    Rh = np_transpose(P)
    same(R.to_host(), Rh)
    rp, col, val = oracle.spgemm(A, P)
    AP = HostCSR(A.nrows, P.ncols, rp, col, val)
    crp, ccol, cval = oracle.spgemm(Rh, AP)
    got = Ac.to_host()
    assert_same_structure(got.rowptr, got.col, crp, ccol)
    assert_close(got.val, cval, oracle.absbound(Rh, AP, crp, ccol))


def test_device_hierarchy_matches_host_restatement(cuda):
    A0 = nb.gen.stencil(15, npts=27)
    levs, Ac = amg.hierarchy(A0, (15, 15, 15), levels=3)
    A, grid = A0, (15, 15, 15)
    for Ad, Pd, Rd, APd in levs:
        same(Ad, A)
        Pt, grid = amg._tentative(*grid)
        P = np_sa_prolongator(A, Pt, 2.0 / 3.0)
        same(Pd, P)
        same(Rd, np_transpose(P))
        rp, col, val = oracle.spgemm(A, P)
        same(APd, HostCSR(A.nrows, P.ncols, rp, col, val))
        crp, ccol, cval = oracle.spgemm(Rd, APd)
        A = HostCSR(Rd.nrows, APd.ncols, crp, ccol, cval)
    same(Ac, A)
