"""The product against the reference's own nsp_spgemm_kernel_hash, both run
on the GPU: the golden fixtures, plus live seeded cases that are checked on
the CPU first to stay clear of the reference paths that can hang or that
miscount (see tests/golden/make_golden.py)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import nsp_b200 as nb
import oracle

from conftest import assert_close, assert_same_structure
from test_golden_cpu import FILES, load

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(oracle.REF_SO):
        pytest.skip("oracle/_ref/libnsp_ref.so not built (reference sources absent)")
    lib = C.CDLL(oracle.REF_SO)
    lib.ref_nsp_spgemm_host.restype = C.c_int
    lib.ref_nsp_spgemm_host.argtypes = [C.c_int] * 3 + [C.c_void_p] * 6 + [C.c_void_p] * 4
    lib.ref_free.argtypes = [C.c_void_p]
    return lib


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_product_matches_golden(cuda, path):
    A, B, (rp, col, val) = load(path)
    got = nb.spgemm(A.to_device(), B.to_device()).to_host()
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert_close(got.val, val, oracle.absbound(A, B, rp, col))


@pytest.mark.parametrize("seed", [101, 202, 303])
def test_product_matches_reference_live(cuda, ref_lib, seed):
    A = nb.gen.random(400, 3000, 1, 30, seed=seed)
    B = nb.gen.random(3000, 6000, 1, 35, seed=seed + 1)
    ok, why = make_golden.reference_bins_safe(A, B)
    assert ok, why
    rp, col, val = make_golden.run_reference(ref_lib, A, B)
    got = nb.spgemm(A.to_device(), B.to_device()).to_host()
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert_close(got.val, val, oracle.absbound(A, B, rp, col))
