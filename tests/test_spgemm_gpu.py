"""GPU parity of the product against the CPU oracle, through the C ABI.

Structure (row_ptr, col) must be bit-exact everywhere. Values are bit-exact
on the deterministic row-group path (B rows strictly increasing, rows of at
most 512 entries), and within |c - c*| <= 1e-12 * sum_k|a_ik b_kj| on the
block / long-row paths whose shared-memory atomics add in arbitrary order.
"""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def run(A, B, **kw):
    dA, dB = A.to_device(), B.to_device()
    C, st = nb.spgemm(dA, dB, return_stats=True, **kw)
    return C.to_host(), st


def check(A, B, exact=None, **kw):
    """Compare with the oracle; exact=None picks bitwise when every row is on
    the deterministic path."""
    got, st = run(A, B, **kw)
    rp, col, val = oracle.spgemm(A, B)
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert st["nnz"] == rp[-1]
    if exact is None:
        exact = st["b_sorted"] and sum(st["num_bins"][6:]) == 0
    if exact:
        assert_bitwise(got.val, val)
    else:
        assert_close(got.val, val, oracle.absbound(A, B, rp, col))
    return got, st


def test_stencil7_32_bitexact(cuda):
    A = nb.gen.stencil(32, npts=7)
    got, st = check(A, A, exact=True)
    assert st["intprod"] == 1_526_528 and st["nnz"] == 776_576


@pytest.mark.parametrize("L", [3, 11, 24])
def test_stencil27_bitexact(cuda, L):
    A = nb.gen.stencil(L, npts=27)
    check(A, A, exact=True)


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_group_lanes_agree(cuda, lanes):
    A = nb.gen.random(3000, 2500, 0, 60, seed=11)
    B = nb.gen.random(2500, 2000, 0, 40, seed=12)
    check(A, B, group_lanes=lanes)


def test_powerlaw_small_all_paths(cuda):
    P = nb.gen.powerlaw(40_000, max_deg=8000, seed=3)
    got, st = check(P, P)
    assert sum(st["num_bins"][6:]) > 0  # block and long kernels exercised


def test_every_bin(cuda):
    # rows whose degrees sweep 0..2^13 against a B with 16 entries per row
    n = 3000
    deg = np.minimum((1.35 ** (np.arange(n) % 40)).astype(np.int64), 2600)
    deg[::97] = 0
    rng = np.random.default_rng(1)
    ncols = 2600
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(deg)
    col = np.concatenate([np.sort(rng.choice(ncols, d, replace=False)) for d in deg]).astype(np.int32)
    A = HostCSR(n, ncols, rp, col, rng.uniform(-1, 1, len(col)))
    B = nb.gen.random(ncols, 40_000, 16, 16, seed=9)
    got, st = check(A, B)
    assert sum(1 for c in st["sym_bins"] if c) >= 8
    assert sum(1 for c in st["num_bins"] if c) >= 7


def test_heaviest_rows_last(cuda):
    # A-row degrees rising with the row index: every block-per-row list is
    # reordered heaviest first before its launch (symbolic bins 8-11, numeric
    # bins 6-9)
    n, ncols = 1200, 3000
    deg = np.linspace(0, 2600, n).astype(np.int64)
    rng = np.random.default_rng(5)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(deg)
    col = np.concatenate([np.sort(rng.choice(ncols, d, replace=False)) for d in deg]).astype(np.int32)
    A = HostCSR(n, ncols, rp, col, rng.uniform(-1, 1, len(col)))
    B = nb.gen.random(ncols, 60_000, 16, 16, seed=6)
    got, st = check(A, B)
    assert all(st["num_bins"][b] > 1 for b in (6, 7, 8, 9))
    assert sum(st["sym_bins"][8:]) > 1


def test_long_rows_wide_column_space(cuda):
    # B with more than 2^18 columns: the long-row kernel runs one block per SM
    # (64 registers a thread) with a bitmap over all 500,000 columns; 927 rows
    # of more than 6,144 entries add into C.val with fp64 atomics, and row 0
    # (1.6 M products, 480 k entries) shares the launch with them
    rng = np.random.default_rng(8)
    n, k, m = 1500, 300_000, 500_000
    deg = rng.integers(0, 2000, n)
    deg[0] = 200_000
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(deg)
    col = np.concatenate([np.sort(rng.choice(k, d, replace=False)) for d in deg]).astype(np.int32)
    A = HostCSR(n, k, rp, col, rng.uniform(-1, 1, len(col)))
    B = nb.gen.random(k, m, 4, 12, seed=9)
    got, st = check(A, B)
    assert st["num_bins"][9] > 100


def test_block_bin_longer_than_order_cap(cuda):
    # 36,000 rows in numeric bin 6 (513..1024 entries), more than the 32,768
    # rows a list may hold to be reordered, so that list stays in row order;
    # 4,000 short rows make a second bin, so the rows are permuted at all
    long_rows = nb.gen.random(36_000, 100_000, 40, 40, seed=31)
    short_rows = nb.gen.random(4_000, 100_000, 4, 4, seed=33)
    rp = np.concatenate([long_rows.rowptr, short_rows.rowptr[1:] + long_rows.nnz]).astype(np.int32)
    A = HostCSR(40_000, 100_000, rp, np.concatenate([long_rows.col, short_rows.col]),
                np.concatenate([long_rows.val, short_rows.val]))
    B = nb.gen.random(100_000, 1_000_000, 16, 16, seed=32)
    got, st = check(A, B)
    assert st["num_bins"][6] > 32_768 and sum(st["num_bins"][:6]) > 0


def test_rectangular_and_empty_rows(cuda):
    A = nb.gen.random(1000, 50, 0, 3, seed=4)   # many empty rows
    B = nb.gen.random(50, 10_000, 0, 2, seed=5)
    check(A, B)


def test_empty_matrices(cuda):
    z = HostCSR(0, 5, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = nb.gen.random(5, 7, 1, 3, seed=1)
    got, st = run(z, B)
    assert got.nrows == 0 and got.nnz == 0 and list(got.rowptr) == [0]
    A = HostCSR(4, 5, np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0))
    got, st = run(A, B)
    assert list(got.rowptr) == [0] * 5 and got.nnz == 0


def test_single_column_and_dense_row(cuda):
    A = nb.gen.random(300, 1, 1, 1, seed=2)
    B = nb.gen.random(1, 5000, 5000, 5000, seed=3)   # one dense B row
    check(A, B)


def test_unsorted_and_duplicate_b_rows(cuda):
    rng = np.random.default_rng(7)
    A = nb.gen.random(2000, 800, 1, 30, seed=21)
    B = nb.gen.random(800, 3000, 1, 30, seed=22)
    col = B.col.copy()
    for i in range(0, B.nrows, 3):  # shuffle every third row, duplicate an entry
        a, b = B.rowptr[i], B.rowptr[i + 1]
        seg = col[a:b]
        rng.shuffle(seg)
        if b - a >= 2:
            seg[0] = seg[-1]
        col[a:b] = seg
    Bu = HostCSR(B.nrows, B.ncols, B.rowptr, col, B.val)
    got, st = check(A, Bu)
    assert st["b_sorted"] == 0


def test_unsorted_long_rows(cuda):
    P = nb.gen.powerlaw(20_000, max_deg=10_000, seed=8)
    rng = np.random.default_rng(3)
    col = P.col.copy()
    for i in range(0, P.nrows, 5):
        a, b = P.rowptr[i], P.rowptr[i + 1]
        rng.shuffle(col[a:b])
    Pu = HostCSR(P.nrows, P.ncols, P.rowptr, col, P.val)
    check(P, Pu)


@pytest.mark.parametrize("shuffle", [False, True])
def test_wide_span_rows(cuda, shuffle):
    # B's columns spread over 3M: the long rows' spans cover several 2^20-column
    # windows, rows of 6K..24K products take the symbolic hash table, rows of
    # 4K..6K entries accumulate in shared memory window by window, longer ones
    # in C.val; shuffled B rows make every span [0, ncols)
    rng = np.random.default_rng(17)
    ncols, nbr, per = 3_000_000, 2000, 25
    pool = np.sort(rng.choice(ncols, 150_000, replace=False))
    bcol = np.concatenate([np.sort(rng.choice(pool, per, replace=False))
                           for _ in range(nbr)]).astype(np.int32)
    brp = (np.arange(nbr + 1) * per).astype(np.int32)
    if shuffle:
        for i in range(nbr):
            rng.shuffle(bcol[brp[i]:brp[i + 1]])
    B = HostCSR(nbr, ncols, brp, bcol, rng.uniform(-1, 1, len(bcol)))
    deg = np.linspace(100, 2000, 60).astype(np.int64)
    arp = np.zeros(len(deg) + 1, np.int32)
    arp[1:] = np.cumsum(deg)
    acol = np.concatenate([np.sort(rng.choice(nbr, d, replace=False)) for d in deg])
    A = HostCSR(len(deg), nbr, arp, acol.astype(np.int32), rng.uniform(-1, 1, int(arp[-1])))
    got, st = check(A, B)
    assert st["b_sorted"] == (0 if shuffle else 1)
    assert sum(st["sym_bins"][8:11]) > 0 and st["sym_bins"][11] > 0
    nz = np.diff(got.rowptr)
    assert np.any((nz > 4096) & (nz <= 6144)) and np.any(nz > 6144)


def test_two_call_matches_one_call(cuda):
    A = nb.gen.random(4000, 3000, 0, 50, seed=31)
    B = nb.gen.random(3000, 3500, 0, 50, seed=32)
    dA, dB = A.to_device(), B.to_device()
    one = nb.spgemm(dA, dB).to_host()
    rp, nnz = nb.spgemm_symbolic(dA, dB)
    two = nb.spgemm_numeric(dA, dB, rp, nnz).to_host()
    assert_same_structure(two.rowptr, two.col, one.rowptr, one.col)
    # rows on the block path add with shared-memory atomics: order may vary
    assert_close(two.val, one.val, oracle.absbound(A, B, one.rowptr, one.col))


def test_caller_provided_output_and_capacity(cuda):
    import torch
    A = nb.gen.stencil(9, npts=27)
    dA = A.to_device()
    ref = nb.spgemm(dA, dA).to_host()
    out = nb.DeviceCSR(A.nrows, A.ncols, torch.empty(A.nrows + 1, dtype=torch.int32, device="cuda"),
                       torch.empty(ref.nnz + 10, dtype=torch.int32, device="cuda"),
                       torch.empty(ref.nnz + 10, dtype=torch.float64, device="cuda"))
    got = nb.spgemm(dA, dA, out=out).to_host()
    assert_bitwise(got.val, ref.val)
    small = nb.DeviceCSR(A.nrows, A.ncols, out.rowptr, out.col[:5], out.val[:5])
    with pytest.raises(nb.NspbError) as e:
        nb.spgemm(dA, dA, out=small)
    assert e.value.status == nb._lib.ERR_CAPACITY


def test_invalid_arguments(cuda):
    A = nb.gen.random(10, 20, 1, 3, seed=1).to_device()
    B = nb.gen.random(21, 5, 1, 3, seed=2).to_device()
    with pytest.raises(nb.NspbError) as e:
        nb.spgemm(A, B)
    assert e.value.status == nb._lib.ERR_INVALID


def test_deterministic_repeats(cuda):
    A = nb.gen.stencil(14, npts=27)
    dA = A.to_device()
    first = nb.spgemm(dA, dA).to_host()
    for _ in range(5):
        again = nb.spgemm(dA, dA).to_host()
        assert_same_structure(again.rowptr, again.col, first.rowptr, first.col)
        assert_bitwise(again.val, first.val)


def test_intprod_matches_oracle(cuda):
    P = nb.gen.powerlaw(30_000, max_deg=3000, seed=4)
    row, tot = nb.intprod(P.to_device(), P.to_device())
    oref, otot = oracle.intprod(P, P)
    assert tot == otot
    np.testing.assert_array_equal(row.cpu().numpy(), oref)


def test_sfcsr_shim_and_version1(cuda):
    A = nb.gen.stencil(10, npts=27)
    B = nb.gen.random(A.ncols, 900, 1, 20, seed=3)
    dA, dB = A.to_device(), B.to_device()
    a, b, c = nb.sfcsr_of(dA), nb.sfcsr_of(dB), nb.SfCSR()
    nb.nsp_spgemm_kernel_hash(a, b, c)
    assert c.M == A.nrows and c.N == B.ncols
    C = nb.DeviceCSR(c.M, c.N, nb.adopt(c.d_rpt, c.M + 1, "int32"),
                     nb.adopt(c.d_col, c.nnz, "int32"), nb.adopt(c.d_val, c.nnz, "float64"))
    h = C.to_host()
    rp, col, val = oracle.spgemm(A, B)
    assert_same_structure(h.rowptr, h.col, rp, col)
    assert_bitwise(h.val, val)
    C2, loc = nb.nsparseMGPU_version1(dA, dB)
    assert loc > 0
    assert_bitwise(C2.to_host().val, val)


def test_stencil27_128_full_size_properties(cuda):
    """The benchmark workload at full size: closed-form row counts, the total
    sum 1^T A A 1, and sampled row blocks against the oracle."""
    import torch
    L = 128
    A = nb.gen.stencil(L, npts=27)
    dA = A.to_device()
    C, st = nb.spgemm(dA, dA, return_stats=True)
    assert st["nnz"] == (5 * L - 6) ** 3 and st["intprod"] == (9 * L - 10) ** 3
    # per-row count = product of per-dimension band widths
    w = np.array([min(i + 2, L - 1) - max(i - 2, 0) + 1 for i in range(L)], np.int64)
    cnt = (w[None, None, :] * w[None, :, None] * w[:, None, None]).ravel()
    rp = C.rowptr.cpu().numpy()
    np.testing.assert_array_equal(np.diff(rp), cnt)
    # 1^T C 1 = (A^T 1) . (A 1)
    S = A.to_scipy()
    ones = np.ones(A.nrows)
    ref_sum = float((S.T @ ones) @ (S @ ones))
    got_sum = float(C.val.sum().item())
    assert abs(got_sum - ref_sum) <= 1e-9 * abs(ref_sum)
    # three row blocks bit-exact against the oracle
    for r0 in (0, A.nrows // 2 - 700, A.nrows - 1500):
        r1 = r0 + 1500
        brp, bcol, bval = oracle.spgemm_rows(A, A, r0, r1)
        a, b = int(rp[r0]), int(rp[r1])
        np.testing.assert_array_equal(rp[r0:r1 + 1] - a, brp)
        np.testing.assert_array_equal(C.col[a:b].cpu().numpy(), bcol)
        assert_bitwise(C.val[a:b].cpu().numpy(), bval)
    del C
    torch.cuda.empty_cache()


@pytest.mark.parametrize("kind", ["sorted", "shuffled", "duplicate"])
def test_same_operand_order_check(cuda, kind):
    # A·A with one device matrix: the order of B (= A) is checked by the row
    # walk that counts the intermediate products instead of a separate pass;
    # rows of more than 1024 entries (counted by a block each) included, and
    # the duplicate goes into the longest row
    P = nb.gen.powerlaw(6000, max_deg=3000, seed=13)
    assert np.diff(P.rowptr).max() > 1024
    col = P.col.copy()
    rng = np.random.default_rng(5)
    if kind == "shuffled":
        for i in range(0, P.nrows, 7):
            rng.shuffle(col[P.rowptr[i]:P.rowptr[i + 1]])
    elif kind == "duplicate":
        i = int(np.argmax(np.diff(P.rowptr)))
        col[P.rowptr[i] + 1] = col[P.rowptr[i]]  # a repeated column breaks strict order
    M = HostCSR(P.nrows, P.ncols, P.rowptr, col, P.val)
    d = M.to_device()
    C, st = nb.spgemm(d, d, return_stats=True)
    assert st["b_sorted"] == (1 if kind == "sorted" else 0)
    got = C.to_host()
    rp, ocol, val = oracle.spgemm(M, M)
    assert_same_structure(got.rowptr, got.col, rp, ocol)
    assert_close(got.val, val, oracle.absbound(M, M, rp, ocol))
