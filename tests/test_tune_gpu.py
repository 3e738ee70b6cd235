"""The autotuner's knobs (threads per row, numeric table size) and the
autotuner itself: every candidate is a valid, bit-exact configuration."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle

from conftest import assert_bitwise, assert_same_structure

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lanes", [8, 16, 32])
@pytest.mark.parametrize("shift", [0, 1])
def test_knobs_bitexact(cuda, lanes, shift):
    A = nb.gen.random(3000, 2500, 0, 60, seed=21)
    B = nb.gen.random(2500, 2000, 0, 9, seed=22)
    C, st = nb.spgemm(A.to_device(), B.to_device(), group_lanes=lanes, table_shift=shift,
                      return_stats=True)
    rp, col, val = oracle.spgemm(A, B)
    h = C.to_host()
    assert_same_structure(h.rowptr, h.col, rp, col)
    assert sum(st["num_bins"][6:]) == 0  # every row on the row-group path
    assert_bitwise(h.val, val)


def test_autotune_picks_a_measured_candidate(cuda):
    A = nb.gen.stencil(24, npts=27)
    dA = A.to_device()
    best, report = nb.autotune(dA, dA, reps=2)
    assert len(report) == 6 and all(ms > 0 for _, _, ms in report)
    fastest = min(report, key=lambda r: r[2])
    assert (best["group_lanes"], best["table_shift"]) == fastest[:2]
    C = nb.spgemm(dA, dA, group_lanes=best["group_lanes"], table_shift=best["table_shift"])
    rp, col, val = oracle.spgemm(A, A)
    h = C.to_host()
    assert_same_structure(h.rowptr, h.col, rp, col)
    assert_bitwise(h.val, val)
