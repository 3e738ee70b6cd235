"""nspb_spgemm_noalloc: the product for callers that may not allocate memory
during the call (their framework owns every device byte, or the memory was
reserved up front). It takes C's arrays from the caller and its scratch from
a fixed device array inside the library.

Checked here through the C ABI: two calls in a row give the same C as the
allocating entry point nspb_spgemm (structure bit-exact; values bit-exact on
the deterministic row-group path, else within 1e-12 of sum|a b|), and an A
with more rows than the fixed scratch holds is rejected up front. The file
is named to be collected last, and each test builds its own inputs, so it
passes alone in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import nsp_b200 as nb
import oracle
from nsp_b200 import _lib
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu

_fn = nb.lib.nspb_spgemm_noalloc
_fn.restype = C.c_int
_fn.argtypes = [C.POINTER(_lib.CsrIn), C.POINTER(_lib.CsrIn), C.POINTER(_lib.CsrOut),
                C.POINTER(_lib.Opts), C.POINTER(_lib.Stats)]


def noalloc_product(dA, dB, capacity):
    """One nspb_spgemm_noalloc call into freshly preallocated tensors."""
    rowptr = torch.full((dA.nrows + 1,), -7, dtype=torch.int32, device="cuda")
    col = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device="cuda")
    val = torch.full((max(capacity, 1),), float("nan"), dtype=torch.float64, device="cuda")
    a, b = dA.as_in(), dB.as_in()
    c = _lib.CsrOut()
    c.rowptr, c.col, c.val = rowptr.data_ptr(), col.data_ptr(), val.data_ptr()
    c.capacity = capacity
    o = nb.make_opts(check_errors=True)
    st = _lib.Stats()
    status = _fn(C.byref(a), C.byref(b), C.byref(c), C.byref(o), C.byref(st))
    torch.cuda.synchronize()
    return status, c.nnz, rowptr, col, val, st


CASES = {
    "stencil27_30": lambda: (nb.gen.stencil(30, npts=27),) * 2,
    "powerlaw_40k": lambda: (nb.gen.powerlaw(40_000, max_deg=8000, seed=3),) * 2,
    "random_rect": lambda: (nb.gen.random(5000, 4000, 0, 60, seed=11),
                            nb.gen.random(4000, 3000, 0, 40, seed=12)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_spgemm_twice(cuda, name):
    A, B = CASES[name]()
    dA, dB = A.to_device(), B.to_device()
    ref, rst = nb.spgemm(dA, dB, return_stats=True)
    ref = ref.to_host()
    orp, ocol, _ = oracle.spgemm(A, B)
    assert_same_structure(ref.rowptr, ref.col, orp, ocol)  # and both against the oracle
    deterministic = rst["b_sorted"] and sum(rst["num_bins"][6:]) == 0
    bound = oracle.absbound(A, B, ref.rowptr, ref.col)
    for _ in range(2):  # the second call sees the first call's scratch contents
        status, nnz, rowptr, col, val, st = noalloc_product(dA, dB, ref.nnz + 3)
        assert status == _lib.OK, nb.lib.nspb_strerror(status)
        assert nnz == ref.nnz and st.nnz == ref.nnz
        assert_same_structure(rowptr.cpu().numpy(), col[:nnz].cpu().numpy(), ref.rowptr, ref.col)
        if deterministic:
            assert_bitwise(val[:nnz].cpu().numpy(), ref.val)
        else:
            assert_close(val[:nnz].cpu().numpy(), ref.val, bound)


def test_noalloc_takes_no_device_memory(cuda):
    """After a warm-up call (which reserves the fixed array and loads the
    kernels), a call leaves the device's free memory unchanged, and its result
    equals the oracle's."""
    A = nb.gen.stencil(24, npts=27, seed=4)
    dA = A.to_device()
    rp, col, val = oracle.spgemm(A, A)
    cap = len(col)
    rowptr = torch.empty(A.nrows + 1, dtype=torch.int32, device="cuda")
    ccol = torch.empty(cap, dtype=torch.int32, device="cuda")
    cval = torch.empty(cap, dtype=torch.float64, device="cuda")
    a = dA.as_in()
    c = _lib.CsrOut()
    c.rowptr, c.col, c.val = rowptr.data_ptr(), ccol.data_ptr(), cval.data_ptr()
    c.capacity = cap
    o = nb.make_opts(check_errors=True)

    def call():
        status = _fn(C.byref(a), C.byref(a), C.byref(c), C.byref(o), None)
        torch.cuda.synchronize()
        assert status == _lib.OK, nb.lib.nspb_strerror(status)
    call()  # warm-up
    free0 = torch.cuda.mem_get_info()[0]
    call()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0
    assert_same_structure(rowptr.cpu().numpy(), ccol.cpu().numpy(), rp, col)
    assert_bitwise(cval.cpu().numpy(), val)


def test_noalloc_capacity_reported(cuda):
    A = nb.gen.stencil(10, npts=27)
    dA = A.to_device()
    status, nnz, *_ = noalloc_product(dA, dA, 100)
    assert status == _lib.ERR_CAPACITY
    assert nnz == (5 * 10 - 6) ** 3


def test_noalloc_rejects_more_rows_than_its_scratch(cuda):
    n = 4_300_000  # past the ~4.19 million rows the fixed scratch holds
    A = HostCSR(n, 8, np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = HostCSR(8, 8, np.zeros(9, np.int32), np.zeros(0, np.int32), np.zeros(0))
    status, nnz, *_ = noalloc_product(A.to_device(), B.to_device(), 16)
    assert status == _lib.ERR_CAPACITY
    assert nnz == -1  # told apart from "C too small", which reports the size needed
    ok = HostCSR(4_000_000, 8, np.zeros(4_000_001, np.int32), np.zeros(0, np.int32),
                 np.zeros(0))
    status, nnz, rowptr, *_ = noalloc_product(ok.to_device(), B.to_device(), 16)
    assert status == _lib.OK and nnz == 0
    assert int(rowptr.max().item()) == 0
