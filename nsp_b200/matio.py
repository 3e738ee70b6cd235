"""Matrix files in the reference's formats, through the library's C readers
and writers (include/nspb.h, "matrix files"):

  read_coo_bin(path, header_type=1, index_bytes=8)  src/READ_MATRIX_MPI.cpp:146-356
  read_coo_ascii(path)                               src/READ_MATRIX_MPI.cpp:365
  write_coo_bin(path, M, index_bytes=8)              main.cu:468-512
  write_mtx(path, M)                                 src/matrixIO.cu:299-339

Readers follow load_MatrixMPI on one rank (src/distribute.cu:1071-1125): local
row 0 is the first row holding an entry (`first_row` gives its file row), and
out-of-order rows are stably sorted by column.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import HostCsr, check, lib
from .csr import HostCSR


def _adopt(h: HostCsr):
    n, nnz = int(h.nrows), int(h.nnz)
    try:
        rp = np.ctypeslib.as_array(C.cast(h.rowptr, C.POINTER(C.c_int32)), (n + 1,)).copy()
        col = (np.ctypeslib.as_array(C.cast(h.col, C.POINTER(C.c_int32)), (nnz,)).copy()
               if nnz else np.zeros(0, np.int32))
        val = (np.ctypeslib.as_array(C.cast(h.val, C.POINTER(C.c_double)), (nnz,)).copy()
               if nnz else np.zeros(0, np.float64))
    finally:
        lib.nspb_host_csr_free(C.byref(h))
    M = HostCSR(n, int(h.ncols), rp, col, val)
    return M, {"full_nrows": int(h.full_nrows), "first_row": int(h.first_row)}


def read_coo_bin(path, header_type: int = 1, index_bytes: int = 8, info: bool = False):
    h = HostCsr()
    check(lib.nspb_read_coo_bin(os.fsencode(path), int(header_type), int(index_bytes),
                                C.byref(h)), f"nspb_read_coo_bin({path})")
    M, meta = _adopt(h)
    return (M, meta) if info else M


def read_coo_ascii(path, info: bool = False):
    h = HostCsr()
    check(lib.nspb_read_coo_ascii(os.fsencode(path), C.byref(h)), f"nspb_read_coo_ascii({path})")
    M, meta = _adopt(h)
    return (M, meta) if info else M


def _arrays(M: HostCSR):
    rp = np.ascontiguousarray(M.rowptr, np.int32)
    col = np.ascontiguousarray(M.col, np.int32)
    val = np.ascontiguousarray(M.val, np.float64)
    return rp, col, val


def write_coo_bin(path, M: HostCSR, index_bytes: int = 8) -> None:
    rp, col, val = _arrays(M)
    check(lib.nspb_write_coo_bin(os.fsencode(path), rp.ctypes.data, col.ctypes.data,
                                 val.ctypes.data, M.nrows, M.ncols, int(index_bytes)),
          f"nspb_write_coo_bin({path})")


def write_mtx(path, M: HostCSR) -> None:
    rp, col, val = _arrays(M)
    check(lib.nspb_write_mtx(os.fsencode(path), rp.ctypes.data, col.ctypes.data,
                             val.ctypes.data, M.nrows, M.ncols), f"nspb_write_mtx({path})")
