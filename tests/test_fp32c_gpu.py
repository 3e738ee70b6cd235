"""FP32 two-sum compensated mode against the fp64 oracle on the same
(fp32-representable) values: structure bit-exact, |c - c*| <= 1e-10 *
sum_k|a_ik b_kj| (the target), and rows accumulated in fp64 instead (their
a-priori bound above the tolerance) bit-exact on the deterministic path."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def as32(h):
    return HostCSR(h.nrows, h.ncols, h.rowptr, h.col, h.val.astype(np.float32))


def run32(A, B, **kw):
    C, st = nb.spgemm(as32(A).to_device(), as32(B).to_device(), precision="fp32c",
                      return_stats=True, **kw)
    return C.to_host(), st


def max_scaled_err(val, ref, bound):
    return float(np.max(np.abs(val - ref) / np.maximum(bound, 1e-300))) if len(val) else 0.0


def test_fp32c_stencil27(cuda):
    A = nb.gen.stencil(20, npts=27, fp32=True)
    got, st = run32(A, A)
    rp, col, val = oracle.spgemm(A, A)
    assert_same_structure(got.rowptr, got.col, rp, col)
    bound = oracle.absbound(A, A, rp, col)
    assert_close(got.val, val, bound, tol=1e-10)
    err = max_scaled_err(got.val, val, bound)
    print(f"stencil27 20^3 fp32c: max |c-c*|/sum|ab| = {err:.3e}, bound {st['max_row_err']:.3e}")
    assert st["rows_redone"] == 0
    assert 0 < st["max_row_err"] <= 1e-10
    assert err <= st["max_row_err"] + 1e-15


def test_fp32c_powerlaw_mixed_rows(cuda):
    P = nb.gen.powerlaw(30_000, max_deg=3000, seed=9, fp32=True)
    got, st = run32(P, P)
    rp, col, val = oracle.spgemm(P, P)
    assert_same_structure(got.rowptr, got.col, rp, col)
    bound = oracle.absbound(P, P, rp, col)
    assert_close(got.val, val, bound, tol=1e-10)
    assert st["rows_redone"] > 0  # long rows went to fp64
    print(f"powerlaw fp32c: max err {max_scaled_err(got.val, val, bound):.3e}, "
          f"rows in fp64 {st['rows_redone']}")


def test_fp32c_tight_tolerance_is_fp64(cuda):
    A = nb.gen.stencil(9, npts=27, fp32=True)
    got, st = run32(A, A, comp_tol=1e-15)  # no row qualifies for fp32 pairs
    rp, col, val = oracle.spgemm(A, A)
    assert st["rows_redone"] == A.nrows
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert_bitwise(got.val, val)  # fp32 products are exact in fp64; A-row order sums


def test_fp32c_rejects_fp64_inputs(cuda):
    A = nb.gen.stencil(5, npts=27).to_device()
    with pytest.raises(nb.NspbError):
        nb.spgemm(A, A, precision="fp32c")


@pytest.mark.parametrize("case", ["stencil27", "random"])
def test_fp32w_is_exact_fp64_accumulation(cuda, case):
    """fp32 inputs with fp64 accumulation: every product of two fp32 values is
    exact in fp64, so the result equals the fp64 oracle on the widened values
    bit for bit (row-group path), within 1e-12 of sum|ab| everywhere."""
    if case == "stencil27":
        A = B = nb.gen.stencil(16, npts=27, fp32=True)
    else:
        A = nb.gen.random(3000, 2500, 1, 30, seed=4, fp32=True)
        B = nb.gen.random(2500, 4000, 1, 40, seed=5, fp32=True)
    C, st = nb.spgemm(as32(A).to_device(), as32(B).to_device(), precision="fp32w",
                      return_stats=True)
    got = C.to_host()
    rp, col, val = oracle.spgemm(A, B)
    assert_same_structure(got.rowptr, got.col, rp, col)
    if sum(st["num_bins"][6:]) == 0:
        assert_bitwise(got.val, val)
    else:
        assert_close(got.val, val, oracle.absbound(A, B, rp, col))


def test_fp32w_rejects_fp64_inputs(cuda):
    A = nb.gen.stencil(5, npts=27).to_device()
    with pytest.raises(nb.NspbError):
        nb.spgemm(A, A, precision="fp32w")

