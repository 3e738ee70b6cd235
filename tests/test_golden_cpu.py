"""The oracle against fixtures produced by the reference's own
nsp_spgemm_kernel_hash on a B200 (tests/golden/make_golden.py): row_ptr and
col bit-exact, values within 1e-12 * sum_k|a_ik b_kj| (the reference adds
with shared-memory atomics, so its summation order varies)."""
import glob
import os

import numpy as np
import pytest

import oracle
from nsp_b200.csr import HostCSR

from conftest import assert_close, assert_same_structure

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(path):
    z = np.load(path)
    A = HostCSR(int(z["a_shape"][0]), int(z["a_shape"][1]), z["a_rp"], z["a_col"], z["a_val"])
    B = HostCSR(int(z["b_shape"][0]), int(z["b_shape"][1]), z["b_rp"], z["b_col"], z["b_val"])
    return A, B, (z["c_rp"], z["c_col"], z["c_val"])


def test_fixtures_present():
    assert len(FILES) >= 5, "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_matches_reference(path):
    A, B, (rp, col, val) = load(path)
    orp, ocol, oval = oracle.spgemm(A, B)
    assert_same_structure(orp, ocol, rp, col)
    assert_close(oval, val, oracle.absbound(A, B, orp, ocol))
