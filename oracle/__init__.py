"""TEST INFRASTRUCTURE — Python binding of the CPU oracle (oracle/liboracle.so,
built from oracle/gustavson.c) and of the reference's own nsp product
(oracle/_ref/libnsp_ref.so, built from the reference sources by
`make -C oracle ref`).

Only tests, the smoke check and the benchmark's CPU baseline / reference arm
use this package; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libnsp_ref.so")


def build(ref: bool = False) -> None:
    subprocess.run(["make", "-C", _HERE, "all"] + (["ref"] if ref else []), check=True)


def _load():
    if not os.path.exists(ORACLE_SO):
        build()
    lib = C.CDLL(ORACLE_SO)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    sig = {
        "oracle_max_threads": (C.c_int, []),
        "oracle_intprod": (i64, [i32, vp, vp, vp, vp, C.c_int]),
        "oracle_symbolic": (i64, [i32, i32, vp, vp, vp, vp, vp, C.c_int]),
        "oracle_symbolic_rows": (i64, [i32, i32, i32, vp, vp, vp, vp, vp, C.c_int]),
        "oracle_numeric": (C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int]),
        "oracle_numeric_rows": (C.c_int, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                          C.c_int]),
        "oracle_absbound": (C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int]),
        "oracle_getmct": (i64, [vp, i64, i32, i32, vp]),
        "oracle_compactcol": (i64, [vp, i64, i32, i32, vp]),
        "oracle_shrink_col": (None, [vp, i64, vp, i64, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a):
    return a.ctypes.data if a is not None and a.size else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def intprod(A, B, nthreads=0):
    """Per-row intermediate products (int64) and their total."""
    row = np.empty(A.nrows, dtype=np.int64)
    tot = lib().oracle_intprod(A.nrows, _p(A.rowptr), _p(A.col), _p(B.rowptr), _p(row), nthreads)
    return row, int(tot)


def symbolic(A, B, nthreads=0):
    """Row pointer of C = A·B (the union of B-row patterns per A row)."""
    rp = np.empty(A.nrows + 1, dtype=np.int32)
    nnz = lib().oracle_symbolic(A.nrows, B.ncols, _p(A.rowptr), _p(A.col), _p(B.rowptr),
                                _p(B.col), _p(rp), nthreads)
    if nnz < 0:
        raise RuntimeError(f"oracle_symbolic failed: {nnz}")
    return rp


def spgemm(A, B, nthreads=0):
    """C = A·B as (rowptr, col, val) with the reference's semantics: sorted
    columns, kept zeros, fp64 sums of rounded products in A-row order."""
    rp = symbolic(A, B, nthreads)
    nnz = int(rp[-1])
    col = np.empty(max(nnz, 1), dtype=np.int32)   # never NULL, even when empty
    val = np.empty(max(nnz, 1), dtype=np.float64)
    av, bv = _f64(A.val), _f64(B.val)
    st = lib().oracle_numeric(A.nrows, B.ncols, _p(A.rowptr), _p(A.col), _p(av), _p(B.rowptr),
                              _p(B.col), _p(bv), _p(rp), _p(col), _p(val), nthreads)
    if st:
        raise RuntimeError(f"oracle_numeric failed: {st}")
    return rp, col[:nnz], val[:nnz]


def spgemm_rows(A, B, r0, r1, nthreads=0):
    """Rows [r0, r1) of C = A·B (row pointer starting at 0)."""
    rp = np.empty(r1 - r0 + 1, dtype=np.int32)
    nnz = lib().oracle_symbolic_rows(r0, r1, B.ncols, _p(A.rowptr), _p(A.col), _p(B.rowptr),
                                     _p(B.col), _p(rp), nthreads)
    if nnz < 0:
        raise RuntimeError(f"oracle_symbolic_rows failed: {nnz}")
    col = np.empty(max(int(nnz), 1), dtype=np.int32)
    val = np.empty(max(int(nnz), 1), dtype=np.float64)
    av, bv = _f64(A.val), _f64(B.val)
    st = lib().oracle_numeric_rows(r0, r1, B.ncols, _p(A.rowptr), _p(A.col), _p(av),
                                   _p(B.rowptr), _p(B.col), _p(bv), _p(rp), _p(col), _p(val),
                                   nthreads)
    if st:
        raise RuntimeError(f"oracle_numeric_rows failed: {st}")
    return rp, col[:int(nnz)], val[:int(nnz)]


def absbound(A, B, rp, col, nthreads=0):
    """sum_k |a_ik b_kj| for every entry of C (same layout as col)."""
    out = np.empty(len(col), dtype=np.float64)
    av, bv = _f64(A.val), _f64(B.val)
    st = lib().oracle_absbound(A.nrows, B.ncols, _p(A.rowptr), _p(A.col), _p(av), _p(B.rowptr),
                               _p(B.col), _p(bv), _p(rp), _p(col), _p(out), nthreads)
    if st:
        raise RuntimeError(f"oracle_absbound failed: {st}")
    return out


def getmct(col, first, last):
    col = np.ascontiguousarray(col, dtype=np.int32)
    out = np.empty(max(len(col), 1), dtype=np.int32)
    n = lib().oracle_getmct(_p(col), len(col), first, last, out.ctypes.data)
    return out[:n]


def compactcol(arr, lo, hi):
    arr = np.ascontiguousarray(arr, dtype=np.int32)
    out = np.empty(max(len(arr), 1), dtype=np.int32)
    n = lib().oracle_compactcol(_p(arr), len(arr), lo, hi, out.ctypes.data)
    return out[:n]


def shrink_col(col, cols):
    col = np.ascontiguousarray(col, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    out = np.empty(max(len(col), 1), dtype=np.int32)
    lib().oracle_shrink_col(_p(col), len(col), _p(cols), len(cols), out.ctypes.data)
    return out[:len(col)]


def max_threads() -> int:
    return int(lib().oracle_max_threads())
