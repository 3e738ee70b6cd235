"""Row templates of the entry-map path: a row whose A length, B row lengths
and product columns repeat an earlier row's (up to one shift of every column)
takes that row's count and map in the symbolic pass, and the numeric pass
reuses that row's sort. Parity against the oracle, bit for bit, on inputs that
repeat (stencils, identical products in one batch) and on inputs built to
almost repeat: rows whose lengths all equal their neighbours' but one column
moved, in A or in B, so the template check has to find the difference in the
columns. Templates on and off must give identical bytes."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_same_structure

pytestmark = pytest.mark.gpu

NO_TEMPLATES = 0x10000  # opts.row_kernel bit: row templates off
# opts.row_kernel bits 20..27: rows a group takes in a run, exactly as given.
# The automatic run is shortened for launches with few rows per resident
# group (1: no templates), which these small inputs would be.
RUN16 = 16 << 20


def perturb(M: HostCSR, frac: float, seed: int) -> HostCSR:
    """Moves one column of a fraction of the rows to a column the row does not
    hold, keeping every row's length and order (values kept)."""
    rng = np.random.default_rng(seed)
    rp, col, val = M.rowptr, M.col.copy(), M.val.copy()
    rows = rng.choice(M.nrows, max(1, int(frac * M.nrows)), replace=False)
    for r in rows:
        a, b = int(rp[r]), int(rp[r + 1])
        if b - a == 0 or b - a >= M.ncols:
            continue
        have = set(col[a:b].tolist())
        j = a + int(rng.integers(b - a))
        c = int(rng.integers(M.ncols))
        while c in have:
            c = int(rng.integers(M.ncols))
        seg = col[a:b].copy()
        vs = val[a:b].copy()
        seg[j - a] = c
        order = np.argsort(seg, kind="stable")
        col[a:b] = seg[order]
        val[a:b] = vs[order]
    return HostCSR(M.nrows, M.ncols, rp.copy(), col.astype(np.int32), val)


def product(A, B, **kw):
    C, st = nb.spgemm(A.to_device(), B.to_device(), return_stats=True, **kw)
    return C.to_host(), st


def check(A, B, row_kernel_bits=RUN16, **kw):
    got, st = product(A, B, row_kernel=7 | row_kernel_bits, **kw)
    rp, col, val = oracle.spgemm(A, B)
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert_bitwise(got.val, val)
    assert st["entry_map"] == 1
    off, _ = product(A, B, row_kernel=7 | NO_TEMPLATES, **kw)
    assert np.array_equal(off.rowptr, got.rowptr) and np.array_equal(off.col, got.col)
    assert_bitwise(off.val, got.val)
    return st


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_stencil27(cuda, lanes):
    # lanes 8 and 16: B rows of 27 entries are longer than the group
    A = nb.gen.stencil(18, npts=27)
    check(A, A, group_lanes=lanes)


@pytest.mark.parametrize("run", [2, 5, 64])
def test_run_lengths(cuda, run):
    # rows a group takes in a run (opts.row_kernel bits 20..27)
    A = nb.gen.stencil(15, npts=27)
    P = perturb(A, 0.02, seed=17)
    check(P, P, row_kernel_bits=run << 20)


@pytest.mark.parametrize("L", [12, 40])
def test_automatic_run(cuda, L):
    # the library's own run length: 12^3 gives every group about one row (no
    # templates), 40^3 about ten
    A = nb.gen.stencil(L, npts=27)
    check(A, A, row_kernel_bits=0)


def test_stencil7(cuda):
    A = nb.gen.stencil(30, npts=7)
    check(A, A)


@pytest.mark.parametrize("frac", [0.01, 0.2])
def test_moved_columns_in_a(cuda, frac):
    A = nb.gen.stencil(16, npts=27)
    P = perturb(A, frac, seed=11)
    check(P, A)


@pytest.mark.parametrize("frac", [0.01, 0.2])
def test_moved_columns_in_b(cuda, frac):
    A = nb.gen.stencil(16, npts=27)
    P = perturb(A, frac, seed=12)
    check(A, P)


def test_moved_columns_both(cuda):
    A = nb.gen.stencil(20, npts=27)
    check(perturb(A, 0.05, seed=13), perturb(A, 0.05, seed=14))


def test_shifted_values_differ(cuda):
    # the same pattern in every interior row, values drawn per entry: a
    # template reuses the sort, never the values
    A = nb.gen.stencil(14, npts=27)
    rng = np.random.default_rng(3)
    B = HostCSR(A.nrows, A.ncols, A.rowptr, A.col, rng.uniform(-1, 1, A.nnz))
    check(A, B)


def test_batched_identical_products(cuda, monkeypatch):
    # rows of one launch come from two products with their own B arrays: a
    # template found in one product serves rows of the other
    # entry maps and runs of 16 rows (the batched entry takes its opts from here)
    monkeypatch.setenv("NSPB_ROW_KERNEL", str(7 | RUN16))
    A = nb.gen.stencil(12, npts=27)
    A2 = HostCSR(A.nrows, A.ncols, A.rowptr.copy(), A.col.copy(), A.val * 0.5)
    dA, dA2 = A.to_device(), A2.to_device()
    Cs, st = nb.spgemm_batched([dA, dA2], [dA, dA2], return_stats=True)
    assert st["entry_map"] >= 1
    for (X, Y), C in zip(((A, A), (A2, A2)), Cs):
        h = C.to_host()
        rp, col, val = oracle.spgemm(X, Y)
        assert_same_structure(h.rowptr, h.col, rp, col)
        assert_bitwise(h.val, val)
