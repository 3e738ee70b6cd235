"""The autotuner's knobs (threads per row, kernel family, table size, symbolic
and numeric bin thresholds) and the autotuner itself: every candidate is a
valid, bit-exact configuration."""
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


@pytest.mark.parametrize("row_kernel", [1, 2, 3])
@pytest.mark.parametrize("fills", [(50, 25), (75, 37), (90, 50), (10, 10)])
def test_bin_thresholds_bitexact(cuda, row_kernel, fills):
    """Thresholds only move rows between bins whose kernels hold them."""
    A = nb.gen.random(4000, 3000, 0, 40, seed=31)
    B = nb.gen.random(3000, 2500, 1, 20, seed=32)
    C, st = nb.spgemm(A.to_device(), B.to_device(), row_kernel=row_kernel,
                      sym_fill_pct=fills[0], num_fill_pct=fills[1], return_stats=True)
    rp, col, val = oracle.spgemm(A, B)
    h = C.to_host()
    assert_same_structure(h.rowptr, h.col, rp, col)
    if sum(st["num_bins"][6:]) == 0:
        assert_bitwise(h.val, val)
    else:
        from conftest import assert_close
        assert_close(h.val, val, oracle.absbound(A, B, rp, col))


def test_autotune_picks_a_measured_candidate(cuda):
    A = nb.gen.stencil(24, npts=27)
    dA = A.to_device()
    best, report = nb.autotune(dA, dA, reps=2)
    assert 6 <= len(report) <= 16 and all(ms > 0 for _, ms in report)
    fastest = min(report, key=lambda r: r[1])
    assert best == fastest[0]
    C = nb.spgemm(dA, dA, group_lanes=best["group_lanes"], table_shift=best["table_shift"],
                  row_kernel=best["row_kernel"], sym_fill_pct=best["sym_fill_pct"],
                  num_fill_pct=best["num_fill_pct"])
    rp, col, val = oracle.spgemm(A, A)
    h = C.to_host()
    assert_same_structure(h.rowptr, h.col, rp, col)
    assert_bitwise(h.val, val)
