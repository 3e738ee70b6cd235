"""A product driven by the reference's file formats: A and P read from binary
COO files (as main.cu loads them), C = A·P on the GPU, C written back and
compared with the oracle."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200 import matio

from conftest import assert_bitwise, assert_same_structure

pytestmark = pytest.mark.gpu


def test_files_to_product_to_files(cuda, tmp_path):
    A = nb.gen.stencil(12, npts=27)
    P = nb.gen.random(A.ncols, 400, 1, 6, seed=4)
    matio.write_coo_bin(tmp_path / "A.bin", A)
    matio.write_coo_bin(tmp_path / "P.bin", P)
    a = matio.read_coo_bin(tmp_path / "A.bin")
    p = matio.read_coo_bin(tmp_path / "P.bin")
    C = nb.spgemm(a.to_device(), p.to_device()).to_host()
    matio.write_coo_bin(tmp_path / "AP.bin", C)
    got = matio.read_coo_bin(tmp_path / "AP.bin")
    rp, col, val = oracle.spgemm(A, P)
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert_bitwise(got.val, val)
