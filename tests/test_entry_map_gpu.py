"""Entry maps (opts.row_kernel 7, and 0 when the B rows fill the row groups):
the symbolic pass records each intermediate product's entry index in its row
(k_sym_map), and the numeric row-group bins of at most 256 entries add at
that index with no hash table (k_num_map). Parity against the oracle: the
structure bit for bit, and the values bit for bit on these rows (they sum in
A-row order from 0 + a*b, like the oracle)."""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200 import amg
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def check(A, B, **kw):
    C, st = nb.spgemm(A.to_device(), B.to_device(), return_stats=True, **kw)
    got = C.to_host()
    rp, col, val = oracle.spgemm(A, B)
    assert_same_structure(got.rowptr, got.col, rp, col)
    if sum(st["num_bins"][6:]) == 0:
        assert_bitwise(got.val, val)
    else:  # rows of more than 512 entries add atomically
        assert_close(got.val, val, oracle.absbound(A, B, rp, col))
    return st


@pytest.mark.parametrize("L,npts", [(9, 27), (17, 27), (40, 7), (24, 7)])
def test_stencils(cuda, L, npts):
    A = nb.gen.stencil(L, npts=npts)
    st = check(A, A, row_kernel=7)
    assert st["entry_map"] == 1


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_random_every_lane_width(cuda, lanes):
    # rows of 0..60 A entries over B rows of 0..40: quads and byte steps,
    # chunks of several G A entries, rows past 256 entries (no map)
    A = nb.gen.random(3000, 2500, 0, 60, seed=21)
    B = nb.gen.random(2500, 2000, 0, 40, seed=22)
    st = check(A, B, row_kernel=7, group_lanes=lanes)
    assert st["entry_map"] == 1


def test_quads_and_bytes_mixed(cuda):
    # B rows alternate between 30 and 2 entries: some quads hold 3G products
    # and take words, the others fall back to one byte a product
    rng = np.random.default_rng(5)
    nb_rows, ncols = 400, 900
    deg = np.where(np.arange(nb_rows) % 3 == 0, 2, 30)
    rp = np.zeros(nb_rows + 1, np.int32)
    rp[1:] = np.cumsum(deg)
    col = np.concatenate([np.sort(rng.choice(ncols, d, replace=False)) for d in deg])
    B = HostCSR(nb_rows, ncols, rp, col.astype(np.int32), rng.uniform(-1, 1, len(col)))
    A = nb.gen.random(2000, nb_rows, 1, 40, seed=6)
    st = check(A, B, row_kernel=7)
    assert st["entry_map"] == 1


def test_amg_products(cuda):
    pairs = amg.amg_batch(L=18, levels=3)
    for A, B in pairs:
        check(A, B, row_kernel=7)


def test_batched_products(cuda):
    pairs = amg.amg_batch(L=18, levels=3)
    pairs += amg.random_batch(12, 500, 4000, 4, 32, seed=9)
    import os
    os.environ["NSPB_ROW_KERNEL"] = "7"
    try:
        Cs = nb.spgemm_batched([a.to_device() for a, _ in pairs],
                               [b.to_device() for _, b in pairs])
    finally:
        del os.environ["NSPB_ROW_KERNEL"]
    for (A, B), Cp in zip(pairs, Cs):
        h = Cp.to_host()
        rp, col, val = oracle.spgemm(A, B)
        assert_same_structure(h.rowptr, h.col, rp, col)
        assert_close(h.val, val, oracle.absbound(A, B, rp, col))


def test_map_dropped_when_rows_outgrow_it(cuda):
    # B has 8 columns: every row of C has at most 8 entries, so the symbolic
    # bins (by min(products, columns)) size the map for 8 products a row,
    # while the rows have 80: the call drops the map and stays exact
    rng = np.random.default_rng(3)
    n, kb, nc = 500, 60, 8
    B = nb.gen.random(kb, nc, 4, 4, seed=4)
    rp = np.arange(0, 20 * n + 1, 20, dtype=np.int32)
    col = np.concatenate([np.sort(rng.choice(kb, 20, replace=False)) for _ in range(n)])
    A = HostCSR(n, kb, rp, col.astype(np.int32), rng.uniform(-1, 1, len(col)))
    st = check(A, B, row_kernel=7)
    assert st["entry_map"] == 0


def test_automatic_choice(cuda):
    A = nb.gen.stencil(30, npts=27)  # B rows of about 25 on 32 lanes: maps
    assert check(A, A)["entry_map"] == 1
    R = nb.gen.random(4000, 4000, 2, 6, seed=8)  # B rows of 4 on 32 lanes: no maps
    assert check(R, R)["entry_map"] == 0


def test_plan_replays_from_maps(cuda):
    A = nb.gen.stencil(30, npts=27)
    dA = A.to_device()
    plan = nb.Plan([dA], [dA])
    assert plan.stats["entry_map"] == 1
    dA.val.mul_(-0.5)
    plan.execute()
    rp, col, val = oracle.spgemm(A, A)
    got = plan.C[0].val.cpu().numpy()
    assert_bitwise(got, 0.25 * val)


def _as32(h):
    return HostCSR(h.nrows, h.ncols, h.rowptr, h.col, h.val.astype(np.float32))


@pytest.mark.parametrize("precision", ["fp32c", "fp32w"])
def test_fp32_forms_from_maps(cuda, precision):
    # fp32 values: compensated pairs (fp32c) or exact fp64 products (fp32w),
    # against the fp64 oracle on the same fp32-representable values
    A = nb.gen.stencil(30, npts=27, fp32=True)
    d = _as32(A).to_device()
    C, st = nb.spgemm(d, d, precision=precision, return_stats=True)
    got = C.to_host()
    rp, col, val = oracle.spgemm(A, A)
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert st["entry_map"] == 1
    if precision == "fp32w":  # products exact in fp64, summed in A-row order
        assert_bitwise(got.val, val)
    else:
        bound = oracle.absbound(A, A, rp, col)
        assert_close(got.val, val, bound, tol=1e-10)
        err = float(np.max(np.abs(got.val - val) / np.maximum(bound, 1e-300)))
        assert st["rows_redone"] == 0 and err <= st["max_row_err"] + 1e-15


def test_fp32c_maps_rows_over_the_bound_in_fp64(cuda):
    A = nb.gen.stencil(12, npts=27, fp32=True)
    d = _as32(A).to_device()
    C, st = nb.spgemm(d, d, precision="fp32c", comp_tol=1e-15, row_kernel=7, return_stats=True)
    rp, col, val = oracle.spgemm(A, A)
    got = C.to_host()
    assert_same_structure(got.rowptr, got.col, rp, col)
    assert st["entry_map"] == 1 and st["rows_redone"] == A.nrows
    assert_bitwise(got.val, val)
