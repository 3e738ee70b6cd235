"""The benchmark configurations at their stated sizes, against the oracle over
the whole product (no sampling):

  - power-law n = 1M (Zipf alpha 2.1, mean degree 16, max 50k) A·A, fp64:
    every symbolic and numeric bin, the long-row kernels (column-span bitmaps,
    fp64 reductions into C.val) and int32 totals near their limits;
  - the 6 Galerkin products of the SA-AMG hierarchy of the 27-point stencil
    on 96^3 plus 256 random products (n uniform in [1k, 100k], 4-32 entries a
    row) through one batched call, every product checked;
  - FP32 compensated on the 27-point stencil 160^3 and on the power-law 1M
    matrix against the fp64 oracle: the error figures of each matrix are
    printed.

Structure (row_ptr, col) must be bit-exact; fp64 values within 1e-12 of
sum_k |a_ik b_kj| (and 1e-12 relative away from cancellation); compensated
values within 1e-10 of the same. These paths correspond to the reference's
long-row kernels nsp/src/nsp.cu:1725-1897 and :2038-2151.
"""
import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200 import amg
from nsp_b200.csr import HostCSR

from conftest import assert_close, assert_same_structure

pytestmark = pytest.mark.gpu

SEED = 20261203


def _free():
    import torch
    torch.cuda.empty_cache()


def test_powerlaw_1M_fp64(cuda):
    P = nb.gen.powerlaw(1_000_000, alpha=2.1, mean_deg=16.0, max_deg=50_000, seed=SEED)
    dP = P.to_device()
    C, st = nb.spgemm(dP, dP, return_stats=True)
    assert st["sym_bins"][11] > 0, "no row reached the long symbolic bin"
    assert st["num_bins"][9] > 0, "no row reached the long numeric bin"
    h = C.to_host()
    del C
    _free()
    rp, col, val = oracle.spgemm(P, P)
    assert st["intprod"] == oracle.intprod(P, P)[1]
    assert_same_structure(h.rowptr, h.col, rp, col)
    bound = oracle.absbound(P, P, rp, col)
    assert_close(h.val, val, bound)
    err = float(np.max(np.abs(h.val - val) / np.maximum(bound, 1e-300)))
    print(f"power-law 1M fp64: nnz(C) {len(col)}, intprod {st['intprod']}, "
          f"max |c-c*|/sum|ab| {err:.3e}, bins sym {st['sym_bins']} num {st['num_bins']}")


def test_amg96_plus_256_random_batched(cuda):
    pairs = amg.amg_batch(L=96, levels=4, seed=SEED)
    assert len(pairs) == 6
    pairs += amg.random_batch(256, 1000, 100_000, 4, 32, seed=SEED)
    Cs = nb.spgemm_batched([a.to_device() for a, _ in pairs],
                           [b.to_device() for _, b in pairs])
    assert len(Cs) == len(pairs)
    worst = 0.0
    total_nnz = 0
    for p, ((A, B), Cp) in enumerate(zip(pairs, Cs)):
        h = Cp.to_host()
        rp, col, val = oracle.spgemm(A, B)
        assert (h.nrows, h.ncols) == (A.nrows, B.ncols), p
        assert_same_structure(h.rowptr, h.col, rp, col)
        bound = oracle.absbound(A, B, rp, col)
        assert_close(h.val, val, bound)
        if len(val):
            worst = max(worst, float(np.max(np.abs(h.val - val) / np.maximum(bound, 1e-300))))
        total_nnz += len(col)
    print(f"AMG 96^3 + 256 random, batched: {len(pairs)} products, nnz(C) {total_nnz}, "
          f"max |c-c*|/sum|ab| {worst:.3e}")
    del Cs
    _free()


def _fp32c_check(A, label):
    A32 = HostCSR(A.nrows, A.ncols, A.rowptr, A.col, A.val.astype(np.float32))
    d32 = A32.to_device()
    C, st = nb.spgemm(d32, d32, precision="fp32c", return_stats=True)
    h = C.to_host()
    del C
    _free()
    rp, col, val = oracle.spgemm(A, A)  # fp64 oracle on the same (fp32-representable) values
    assert_same_structure(h.rowptr, h.col, rp, col)
    bound = oracle.absbound(A, A, rp, col)
    assert_close(h.val, val, bound, tol=1e-10)
    err = np.abs(h.val - val)
    scaled = float(np.max(err / np.maximum(bound, 1e-300)))
    # per-entry relative error away from cancellation: the Dot2 bound is
    # relative to sum|ab|, so an entry that cancels to 1e-6 of its sum|ab|
    # can carry 1e-6 relative error at 1e-12 scaled error
    away = np.abs(val) > 1e-3 * bound
    rel = float(np.max(err[away] / np.abs(val[away]))) if away.any() else 0.0
    print(f"{label} fp32c vs fp64 oracle: max |c-c*|/sum|ab| {scaled:.3e}, max relative "
          f"error {rel:.3e} over {int(away.sum())} of {len(val)} entries (|c*| > 1e-3 sum|ab|), "
          f"a-priori bound {st['max_row_err']:.3e}, rows in fp64 {st['rows_redone']}")
    assert scaled <= 1e-10 and rel <= 1e-10
    return st


def test_fp32c_stencil27_160(cuda):
    A = nb.gen.stencil(160, npts=27, seed=SEED, fp32=True)
    st = _fp32c_check(A, "27-point stencil 160^3")
    assert st["intprod"] == 2_924_207_000  # past int32: totals are int64


def test_fp32c_powerlaw_1M(cuda):
    P = nb.gen.powerlaw(1_000_000, alpha=2.1, mean_deg=16.0, max_deg=50_000, seed=SEED,
                        fp32=True)
    st = _fp32c_check(P, "power-law 1M")
    assert st["rows_redone"] > 0  # the long rows accumulate in fp64
