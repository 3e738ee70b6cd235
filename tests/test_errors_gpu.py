"""Status codes of the C ABI on the GPU paths: nnz(C) past int32, a device
error word raised by a kernel's own count check, and an unsupported mode.
Every case is an input the library itself turns into an error."""
import numpy as np
import pytest
import torch

import nsp_b200 as nb
from nsp_b200 import _lib
from nsp_b200.csr import HostCSR

pytestmark = pytest.mark.gpu


def test_nnz_past_int32_is_overflow(cuda):
    # 45,000 rows, each hitting one B row of 48,000 entries: nnz(C) = 2.16e9;
    # the symbolic phase counts it and the call stops before allocating C
    n, m = 45_000, 48_000
    A = HostCSR(n, 1, np.arange(n + 1, dtype=np.int32), np.zeros(n, np.int32), np.ones(n))
    B = HostCSR(1, m, np.array([0, m], np.int32), np.arange(m, dtype=np.int32), np.ones(m))
    with pytest.raises(nb.NspbError) as e:
        nb.spgemm(A.to_device(), B.to_device())
    assert e.value.status == _lib.ERR_OVERFLOW


def test_row_count_disagreement_sets_device_error(cuda):
    # the two-call numeric step with a row pointer one entry short on one row:
    # the kernel finds the row's count differs, writes nothing for it and
    # raises the error word (rows of at most 512 entries: row-group kernels)
    A = nb.gen.random(2000, 1500, 1, 20, seed=31)
    B = nb.gen.random(1500, 1200, 1, 10, seed=32)
    dA, dB = A.to_device(), B.to_device()
    rp, nnz = nb.spgemm_symbolic(dA, dB)
    counts = torch.diff(rp)
    r = int(torch.argmax(counts))
    bad = rp.clone()
    bad[r + 1:] -= 1
    with pytest.raises(nb.NspbError) as e:
        nb.spgemm_numeric(dA, dB, bad, nnz - 1)
    assert e.value.status == _lib.ERR_DEVICE
    good = nb.spgemm_numeric(dA, dB, rp, nnz)  # the library still works afterwards
    assert good.nnz == nnz


def test_galerkin_fp32_is_unsupported(cuda):
    A = nb.gen.stencil(6, npts=27)
    P = nb.gen.random(A.ncols, 30, 1, 3, seed=2)
    dA, dP = A.to_device(), P.to_device()
    dP.val = dP.val.float()
    with pytest.raises(nb.NspbError) as e:
        nb.galerkin(dA, dP)
    assert e.value.status in (_lib.ERR_UNSUPPORTED, _lib.ERR_INVALID)
