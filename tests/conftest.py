import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    return torch.device("cuda:0")


def assert_same_structure(rp, col, rp_ref, col_ref):
    np.testing.assert_array_equal(np.asarray(rp), np.asarray(rp_ref))
    np.testing.assert_array_equal(np.asarray(col), np.asarray(col_ref))


def assert_bitwise(val, val_ref):
    a = np.ascontiguousarray(val, dtype=np.float64).view(np.int64)
    b = np.ascontiguousarray(val_ref, dtype=np.float64).view(np.int64)
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, f"{bad.size} values differ bitwise, first at {bad[:5]}"


def assert_close(val, val_ref, bound, tol=1e-12):
    """|c - c*| <= tol * sum_k |a_ik b_kj| (cancellation-safe), and the
    per-entry relative error |c - c*|/|c*| <= tol wherever |c*| is not tiny
    against its own magnitude bound."""
    val = np.asarray(val, dtype=np.float64)
    val_ref = np.asarray(val_ref, dtype=np.float64)
    err = np.abs(val - val_ref)
    bad = np.nonzero(err > tol * bound)[0]
    assert bad.size == 0, f"{bad.size} values off, worst {err[bad].max()} at {bad[:5]}"
    big = np.abs(val_ref) > 1e-3 * bound
    if big.any():
        rel = err[big] / np.abs(val_ref[big])
        assert rel.max() <= tol, f"max relative error {rel.max()}"
