"""CPU checks of the oracle and the generators (no GPU).

The reference has no tests or golden vectors of its own, so the oracle is
pinned by: closed-form structure counts of the stencil products (derived
here from 1-D Kronecker factors), scipy's sparse product on small cases, and
fixtures produced by the reference's nsp_spgemm_kernel_hash (test_golden_cpu).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import nsp_b200 as nb
import oracle
from nsp_b200.csr import HostCSR


def stencil27_counts(L):
    """(nnz(A), intprod, nnz(A·A)) of the 27-point stencil on L^3.
    Per dimension: nnz = 3L-2, sum of squared degrees = 9L-10, nnz of the
    squared 3-band = 5L-6 (pairs with |i-j| <= 2)."""
    return (3 * L - 2) ** 3, (9 * L - 10) ** 3, (5 * L - 6) ** 3


def test_stencil7_32_counts():
    A = nb.gen.stencil(32, npts=7)
    assert A.nnz == 223_232
    _, tot = oracle.intprod(A, A)
    assert tot == 1_526_528
    rp = oracle.symbolic(A, A)
    assert rp[-1] == 776_576


@pytest.mark.parametrize("L", [2, 3, 8, 17, 40])
def test_stencil27_closed_form(L):
    A = nb.gen.stencil(L, npts=27)
    nnz, ip, nnzc = stencil27_counts(L)
    assert A.nnz == nnz
    assert oracle.intprod(A, A)[1] == ip
    assert oracle.symbolic(A, A)[-1] == nnzc


def test_stencil27_128_counts():
    nnz, ip, nnzc = stencil27_counts(128)
    assert (nnz, ip, nnzc) == (55_742_968, 1_489_355_288, 254_840_104)
    A = nb.gen.stencil(128, npts=27)
    assert A.nnz == nnz
    assert oracle.intprod(A, A)[1] == ip


def test_stencil27_values():
    A = nb.gen.stencil(6, npts=27)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0.0  # symmetric
    off = S - sp.diags(S.diagonal())
    assert np.allclose(S.diagonal(), np.asarray(abs(off).sum(axis=1)).ravel() + 1.0)
    assert np.all(np.abs(off.data) <= 1.0)


def test_fp32_values_are_representable():
    A = nb.gen.stencil(5, npts=27, fp32=True)
    assert np.array_equal(A.val, A.val.astype(np.float32).astype(np.float64))
    P = nb.gen.powerlaw(2000, max_deg=200, fp32=True)
    assert np.array_equal(P.val, P.val.astype(np.float32).astype(np.float64))


def test_powerlaw_shape():
    P = nb.gen.powerlaw(200_000, max_deg=50_000)
    deg = np.diff(P.rowptr)
    assert deg.min() >= 1 and deg.max() <= 50_000
    assert 14.0 < deg.mean() < 18.0
    for i in (0, 17, 1234):
        c = P.col[P.rowptr[i]:P.rowptr[i + 1]]
        assert np.all(np.diff(c) > 0)


def test_generators_deterministic():
    a = nb.gen.powerlaw(5000, max_deg=500, seed=7)
    b = nb.gen.powerlaw(5000, max_deg=500, seed=7)
    c = nb.gen.powerlaw(5000, max_deg=500, seed=8)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.val, b.val)
    assert not np.array_equal(a.val[:100], c.val[:100])


def _scipy_product(A, B):
    C = (A.to_scipy() @ B.to_scipy()).tocsr()
    C.sort_indices()
    return C


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_scipy_random(seed):
    A = nb.gen.random(700, 900, 0, 40, seed=seed)
    B = nb.gen.random(900, 500, 1, 25, seed=seed + 100)
    rp, col, val = oracle.spgemm(A, B)
    C = _scipy_product(A, B)
    np.testing.assert_array_equal(rp, C.indptr)
    np.testing.assert_array_equal(col, C.indices)
    np.testing.assert_allclose(val, C.data, rtol=1e-13, atol=0)


def test_oracle_keeps_cancellation_zeros():
    # row 0 of A: [1, 1]; B rows: [x: 1.0], [x: -1.0] -> C(0, x) = 0 kept
    A = HostCSR(1, 2, np.array([0, 2], np.int32), np.array([0, 1], np.int32),
                np.array([1.0, 1.0]))
    B = HostCSR(2, 3, np.array([0, 1, 2], np.int32), np.array([2, 2], np.int32),
                np.array([1.0, -1.0]))
    rp, col, val = oracle.spgemm(A, B)
    assert list(rp) == [0, 1] and list(col) == [2] and val[0] == 0.0


def test_oracle_sums_duplicates_and_unsorted():
    A = HostCSR(1, 2, np.array([0, 3], np.int32), np.array([1, 0, 1], np.int32),
                np.array([2.0, 3.0, 0.5]))
    B = HostCSR(2, 4, np.array([0, 2, 5], np.int32), np.array([3, 1, 2, 0, 2], np.int32),
                np.array([1.0, 2.0, 4.0, 8.0, 16.0]))
    rp, col, val = oracle.spgemm(A, B)
    assert list(col) == [0, 1, 2, 3]
    # B row 1 = {2: 4+16, 0: 8}; A row = 2.5*Brow1 + 3*Brow0
    np.testing.assert_array_equal(val, [2.5 * 8.0, 3 * 2.0, 2.5 * 20.0, 3 * 1.0])


def test_oracle_row_block_matches_full():
    A = nb.gen.random(500, 400, 0, 30, seed=5)
    B = nb.gen.random(400, 300, 0, 30, seed=6)
    rp, col, val = oracle.spgemm(A, B)
    brp, bcol, bval = oracle.spgemm_rows(A, B, 120, 333)
    a, b = rp[120], rp[333]
    np.testing.assert_array_equal(brp, rp[120:334] - a)
    np.testing.assert_array_equal(bcol, col[a:b])
    np.testing.assert_array_equal(bval, val[a:b])


def test_oracle_remap_helpers():
    rng = np.random.default_rng(0)
    col = rng.integers(0, 1000, 5000).astype(np.int32)
    got = oracle.getmct(col, 200, 599)
    ref = np.unique(col[(col < 200) | (col > 599)])
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(oracle.getmct(col, 1, 0), np.unique(col))
    np.testing.assert_array_equal(oracle.compactcol(col, 200, 599), col[(col < 200) | (col > 599)])
    cols = np.unique(col[::3])
    pos = oracle.shrink_col(col, cols)
    ref = np.searchsorted(cols, col)
    ok = (ref < len(cols)) & (cols[np.minimum(ref, len(cols) - 1)] == col)
    np.testing.assert_array_equal(pos, np.where(ok, ref, -1))
