"""Column remap (getmct / compactcol / shrink) through the C ABI against the
oracle's restatement of the reference (src/getmct.cu, src/compactcol.cu,
src/spspmpi.cu:58-84)."""
import ctypes as C

import numpy as np
import pytest
import torch

import nsp_b200 as nb
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.int32)).cuda()


@pytest.mark.parametrize("n,hi", [(0, 10), (1, 10), (5000, 1000), (3_000_000, 2_000_000)])
def test_getmct(cuda, n, hi):
    rng = np.random.default_rng(n)
    col = rng.integers(0, hi, n).astype(np.int32)
    d = dev(col)
    out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    for first, last in ((hi // 4, hi // 2), (1, 0), (0, hi)):
        cnt = C.c_int64(-1)
        nb._lib.check(nb.lib.nspb_getmct(C.c_void_p(d.data_ptr()), n, first, last,
                                         C.c_void_p(out.data_ptr()), C.byref(cnt), None))
        ref = oracle.getmct(col, first, last)
        assert cnt.value == len(ref)
        np.testing.assert_array_equal(out[:cnt.value].cpu().numpy(), ref)


@pytest.mark.parametrize("n", [0, 7, 4096, 4097, 1_000_003])
def test_compactcol(cuda, n):
    rng = np.random.default_rng(n + 1)
    col = rng.integers(0, 1000, n).astype(np.int32)
    d = dev(col)
    out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    cnt = C.c_int64(-1)
    nb._lib.check(nb.lib.nspb_compactcol(C.c_void_p(d.data_ptr()), n, 250, 749,
                                         C.c_void_p(out.data_ptr()), C.byref(cnt), None))
    ref = oracle.compactcol(col, 250, 749)
    assert cnt.value == len(ref)
    np.testing.assert_array_equal(out[:cnt.value].cpu().numpy(), ref)


def test_shrink_col(cuda):
    rng = np.random.default_rng(3)
    col = rng.integers(0, 100_000, 500_000).astype(np.int32)
    cols = np.unique(col[::7])
    out = torch.empty(len(col), dtype=torch.int32, device="cuda")
    dc, dl = dev(col), dev(cols)
    nb._lib.check(nb.lib.nspb_shrink_col(C.c_void_p(dc.data_ptr()), len(col),
                                         C.c_void_p(dl.data_ptr()), len(cols),
                                         C.c_void_p(out.data_ptr()), None))
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.shrink_col(col, cols))
