"""Generate golden fixtures from the reference's own product.

Runs amavliut/nsp's nsp_spgemm_kernel_hash (compiled for sm_100a from the
reference sources into oracle/_ref/libnsp_ref.so by `make -C oracle ref`) on
small seeded inputs and stores A, B and the reference's C in
<out>/<case>.npz. Needs a GPU; run from the repository root:

    python tests/golden/make_golden.py --out tests/golden

Before a case runs, the reference's bins are recomputed on the CPU from the
oracle's counts, and a case is refused when it would reach
  - numeric bin 9 (rows with more than 3584 entries that are not dense):
    nsp_calculate_value_col_bin_each_tb_chunk_dynamic inserts with an
    unbounded while(1) probe (nsp/src/nsp.cu:1725-1897), or
  - a largest symbolic bin of 3 (max intermediate products in (256, 512]):
    row_nz is then not zeroed before nsp_set_row_nz_bin_each_tb<512> adds
    into it (nsp/src/nsp.cu:464, :584), which inflates nnz(C).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import nsp_b200 as nb  # noqa: E402
import oracle  # noqa: E402
from nsp_b200.csr import HostCSR  # noqa: E402


def cases():
    P = nb.gen.powerlaw(20_000, max_deg=150, seed=41)
    return {
        "lap7_12": (nb.gen.stencil(12, npts=7),) * 2,
        "st27_12": (nb.gen.stencil(12, npts=27, seed=12),) * 2,
        "rand_dense_small": (nb.gen.random(300, 2500, 0, 40, seed=1),
                             nb.gen.random(2500, 2500, 1, 36, seed=2)),
        "rand_rect": (nb.gen.random(300, 8000, 1, 20, seed=3),
                      nb.gen.random(8000, 20000, 1, 40, seed=4)),
        "powerlaw_rows": (P.row_block(0, 200), P),
        "dense_rows": (nb.gen.random(150, 300, 100, 200, seed=5),
                       nb.gen.random(300, 400, 50, 100, seed=6)),
    }


def reference_bins_safe(A, B):
    """Refuse inputs that reach the reference paths named in the header."""
    ip, _ = oracle.intprod(A, B)
    rp = oracle.symbolic(A, B)
    nz = np.diff(rp)
    ncols = B.ncols
    dens = nz / max(ncols, 1) * 100.0
    dense = ((ncols <= 5120) & (dens > 10.0)) | (dens > 30.0)
    if np.any((nz > 3584) & ~dense):
        return False, "numeric bin 9 (chunk_dynamic)"
    lim = [64, 128, 256, 512, 1024, 2048, 4096, 8192, 12288]
    top = int(np.searchsorted(lim, ip.max())) if len(ip) else 0
    if top == 3:
        return False, "largest symbolic bin is 3 (row_nz not zeroed)"
    return True, ""


def run_reference(lib, A, B):
    nnz = C.c_int(0)
    crp, ccol, cval = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    av = np.ascontiguousarray(A.val, np.float64)
    bv = np.ascontiguousarray(B.val, np.float64)
    rc = lib.ref_nsp_spgemm_host(A.nrows, A.ncols, B.ncols, A.rowptr.ctypes.data,
                                 A.col.ctypes.data, av.ctypes.data, B.rowptr.ctypes.data,
                                 B.col.ctypes.data, bv.ctypes.data, C.byref(nnz), C.byref(crp),
                                 C.byref(ccol), C.byref(cval))
    if rc:
        raise RuntimeError(f"reference failed with cudaError {rc}")
    n = nnz.value
    rp = np.ctypeslib.as_array(crp, (A.nrows + 1,)).copy()
    col = np.ctypeslib.as_array(ccol, (max(n, 1),))[:n].copy()
    val = np.ctypeslib.as_array(cval, (max(n, 1),))[:n].copy()
    for p in (crp, ccol, cval):
        lib.ref_free(C.cast(p, C.c_void_p))
    return rp, col, val


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    lib = C.CDLL(oracle.REF_SO)
    lib.ref_nsp_spgemm_host.restype = C.c_int
    lib.ref_nsp_spgemm_host.argtypes = [C.c_int] * 3 + [C.c_void_p] * 6 + [C.c_void_p] * 4
    lib.ref_free.argtypes = [C.c_void_p]
    summary = {}
    for name, (A, B) in cases().items():
        ok, why = reference_bins_safe(A, B)
        if not ok:
            summary[name] = {"skipped": why}
            print(name, "skipped:", why, flush=True)
            continue
        rp, col, val = run_reference(lib, A, B)
        orp, ocol, oval = oracle.spgemm(A, B)
        same = bool(np.array_equal(rp, orp) and np.array_equal(col, ocol))
        err = float(np.max(np.abs(val - oval) / np.maximum(oracle.absbound(A, B, orp, ocol), 1e-300))) \
            if same and len(val) else None
        summary[name] = {"nrows": A.nrows, "nnz_c": int(rp[-1]), "structure_equal_oracle": same,
                         "max_scaled_err_vs_oracle": err}
        print(name, summary[name], flush=True)
        np.savez_compressed(os.path.join(args.out, f"{name}.npz"),
                            a_shape=np.array([A.nrows, A.ncols]), a_rp=A.rowptr, a_col=A.col,
                            a_val=A.val, b_shape=np.array([B.nrows, B.ncols]), b_rp=B.rowptr,
                            b_col=B.col, b_val=B.val, c_rp=rp, c_col=col, c_val=val)
    with open(os.path.join(args.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
