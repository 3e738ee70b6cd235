"""The reference-side integration run for real: a C++ program written against
the reference's own interface (tests/dropin/caller.cpp) builds device CSRs as
CSRm::init does, calls nsparseMGPU_version1 and nsp_spgemm_kernel_hash from
libnspb.so, and frees C as CSRm::free does, including
cusparseDestroyMatDescr(*descr) on the descriptor the shim returns. Its
products are compared with the oracle."""
import os
import subprocess

import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from conftest import assert_bitwise, assert_close, assert_same_structure
from dropin import build_caller

pytestmark = pytest.mark.gpu


def _write(path, M):
    with open(path, "wb") as f:
        np.array([M.nrows, M.ncols, M.nnz], dtype=np.int32).tofile(f)
        np.asarray(M.rowptr, dtype=np.int32).tofile(f)
        np.asarray(M.col, dtype=np.int32).tofile(f)
        np.asarray(M.val, dtype=np.float64).tofile(f)


def _read(path):
    with open(path, "rb") as f:
        n, m, nnz = np.fromfile(f, dtype=np.int32, count=3)
        rp = np.fromfile(f, dtype=np.int32, count=n + 1)
        col = np.fromfile(f, dtype=np.int32, count=nnz)
        val = np.fromfile(f, dtype=np.float64, count=nnz)
    return int(n), int(m), rp, col, val


@pytest.mark.parametrize("case", ["stencil27", "powerlaw"])
def test_cpp_dropin_matches_oracle(cuda, tmp_path, case):
    if case == "stencil27":
        A = B = nb.gen.stencil(20, npts=27, seed=9)
    else:
        A = B = nb.gen.powerlaw(20_000, max_deg=3000, seed=5)
    exe = build_caller(str(tmp_path))
    fa, fb = str(tmp_path / "a.bin"), str(tmp_path / "b.bin")
    _write(fa, A)
    _write(fb, B)
    run = subprocess.run([exe, fa, fb, str(tmp_path / "c")], capture_output=True, text=True,
                         timeout=300)
    assert run.returncode == 0, run.stderr
    fields = run.stdout.split()
    # the shim's NULL descriptor passes through cusparseDestroyMatDescr like a
    # created one (status 0 = CUSPARSE_STATUS_SUCCESS)
    assert fields[2] == "destroy_descr_C" and fields[3] == "0", run.stdout
    assert float(fields[1]) > 0.0  # loc_time
    rp, col, val = oracle.spgemm(A, B)
    bound = oracle.absbound(A, B, rp, col)
    for suffix in (".v1", ".kh"):
        n, m, grp, gcol, gval = _read(str(tmp_path / "c") + suffix)
        assert (n, m) == (A.nrows, B.ncols)
        assert_same_structure(grp, gcol, rp, col)
        if case == "stencil27":  # every row on the deterministic row-group path
            assert_bitwise(gval, val)
        else:
            assert_close(gval, val, bound)
