"""Batched products (one block-diagonal pipeline per group of products)
against the oracle, product by product: the Galerkin products of a small
SA-AMG hierarchy plus independent random products of uneven size."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200 import amg
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def check_pair(got, A, B, exact):
    rp, col, val = oracle.spgemm(A, B)
    h = got.to_host()
    assert (h.nrows, h.ncols) == (A.nrows, B.ncols)
    assert_same_structure(h.rowptr, h.col, rp, col)
    if exact:
        assert_bitwise(h.val, val)
    else:
        assert_close(h.val, val, oracle.absbound(A, B, rp, col))


def test_hierarchy_galerkin_matches_oracle(cuda):
    A0 = nb.gen.stencil(15, npts=27)
    levs, Ac = amg.hierarchy(A0, (15, 15, 15), levels=3)
    assert [l[0].nrows for l in levs] == [15 ** 3, 5 ** 3]
    assert Ac.nrows == 2 ** 3
    for A, P, R, AP in levs:
        np.testing.assert_array_equal(np.diff(P.rowptr) > 0, True)
        # R = P^T and AP = A·P against the oracle
        rp, col, val = oracle.spgemm(A, P)
        assert_same_structure(AP.rowptr, AP.col, rp, col)
        assert_bitwise(AP.val, val)
        S = R.to_scipy()
        assert abs(S - P.to_scipy().T).max() == 0.0


def test_batched_matches_oracle(cuda):
    pairs = amg.amg_batch(L=18, levels=3) + amg.random_batch(12, 300, 3000, 2, 14, seed=5)
    pairs.append((HostCSR(0, 7, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)),
                  nb.gen.random(7, 9, 1, 3, seed=1)))  # an empty product in the middle
    pairs += amg.random_batch(3, 100, 400, 0, 3, seed=8)
    Cs, st = nb.spgemm_batched([a.to_device() for a, _ in pairs],
                               [b.to_device() for _, b in pairs], return_stats=True)
    assert len(Cs) == len(pairs)
    exact = sum(st["num_bins"][6:]) == 0
    for got, (A, B) in zip(Cs, pairs):
        check_pair(got, A, B, exact)


def test_batched_equals_single_calls(cuda):
    pairs = amg.random_batch(6, 2000, 6000, 4, 32, seed=9)
    dA = [a.to_device() for a, _ in pairs]
    dB = [b.to_device() for _, b in pairs]
    Cs = nb.spgemm_batched(dA, dB)
    for got, a, b, (A, B) in zip(Cs, dA, dB, pairs):
        one, st = nb.spgemm(a, b, return_stats=True)
        one = one.to_host()
        h = got.to_host()
        assert_same_structure(h.rowptr, h.col, one.rowptr, one.col)
        if sum(st["num_bins"][6:]) == 0:
            assert_bitwise(h.val, one.val)
        else:  # rows on the block path add atomically, in any order
            assert_close(h.val, one.val, oracle.absbound(A, B, one.rowptr, one.col))


def test_batched_fp32c(cuda):
    pairs = amg.random_batch(5, 1000, 4000, 4, 20, seed=12)
    as32 = lambda h: HostCSR(h.nrows, h.ncols, h.rowptr, h.col,
                             h.val.astype(np.float32).astype(np.float64))
    pairs = [(as32(a), as32(b)) for a, b in pairs]
    f32 = lambda h: HostCSR(h.nrows, h.ncols, h.rowptr, h.col, h.val.astype(np.float32))
    Cs, st = nb.spgemm_batched([f32(a).to_device() for a, _ in pairs],
                               [f32(b).to_device() for _, b in pairs], precision="fp32c",
                               return_stats=True)
    for got, (A, B) in zip(Cs, pairs):
        rp, col, val = oracle.spgemm(A, B)
        h = got.to_host()
        assert_same_structure(h.rowptr, h.col, rp, col)
        assert_close(h.val, val, oracle.absbound(A, B, rp, col), tol=1e-10)
