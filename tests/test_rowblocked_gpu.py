"""Row-blocked product (budgeted device memory for C, host output) against
the oracle; the blocks go through the getmct / gather / shrink remap."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("budget", [50_000, 400_000, 10**12])
def test_rowblocked_stencil(cuda, budget):
    A = nb.gen.stencil(14, npts=27)
    C, nblk = nb.spgemm_rowblocked(A.to_device(), A.to_device(), budget)
    rp, col, val = oracle.spgemm(A, A)
    assert_same_structure(C.rowptr, C.col, rp, col)
    assert_bitwise(C.val, val)
    expect_blocks = 1 if budget >= 12 * len(col) + 4 * A.nrows else 2
    assert nblk >= expect_blocks


def test_rowblocked_rectangular_powerlaw(cuda):
    A = nb.gen.powerlaw(6000, ncols=9000, max_deg=900, seed=4)
    B = nb.gen.random(9000, 20000, 0, 12, seed=5)
    C, nblk = nb.spgemm_rowblocked(A.to_device(), B.to_device(), 300_000)
    rp, col, val = oracle.spgemm(A, B)
    assert nblk > 3
    assert_same_structure(C.rowptr, C.col, rp, col)
    assert_close(C.val, val, oracle.absbound(A, B, rp, col))
