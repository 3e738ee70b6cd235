"""ctypes binding of libnspb.so (the C ABI declared in include/nspb.h).

The shared library is built in-tree (``nsp_b200/libnspb.so``). Importing this
module without it raises ImportError: there is no Python or CPU fallback for
the product.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnspb.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C nsp_b200/csrc` "
        "(or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

# ---- status codes (nspb_status) ----------------------------------------------
OK = 0
ERR_INVALID = -1
ERR_OVERFLOW = -2
ERR_ALLOC = -3
ERR_CUDA = -4
ERR_DEVICE = -5
ERR_NO_DEVICE = -6
ERR_UNSUPPORTED = -7
ERR_CAPACITY = -8
ERR_IO = -9

F64 = 0
F32 = 1
PREC_FP64 = 0
PREC_FP32_COMP = 1
PREC_FP32_WIDE = 2


class CsrIn(C.Structure):
    _fields_ = [("nrows", C.c_int32), ("ncols", C.c_int32), ("nnz", C.c_int64),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p),
                ("val_type", C.c_int32), ("_pad", C.c_int32)]


class CsrOut(C.Structure):
    _fields_ = [("nrows", C.c_int32), ("ncols", C.c_int32), ("nnz", C.c_int64),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p),
                ("capacity", C.c_int64)]


class Opts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("assume_sorted", C.c_int32),
                ("check_errors", C.c_int32), ("group_lanes", C.c_int32),
                ("timing", C.c_int32), ("batch_max_products", C.c_int32),
                ("comp_tol", C.c_double), ("stream", C.c_void_p),
                ("num_table_shift", C.c_int32), ("row_kernel", C.c_int32),
                ("sym_fill_pct", C.c_int32), ("num_fill_pct", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("intprod", C.c_int64), ("nnz", C.c_int64),
                ("sym_bins", C.c_int32 * 16), ("num_bins", C.c_int32 * 16),
                ("rows_redone", C.c_int32), ("b_sorted", C.c_int32),
                ("max_row_err", C.c_double), ("launches", C.c_int32),
                ("ms_rowinfo", C.c_float), ("ms_symbolic", C.c_float),
                ("ms_scan", C.c_float), ("ms_numeric", C.c_float), ("entry_map", C.c_int32)]


class TuneEntry(C.Structure):
    _fields_ = [("group_lanes", C.c_int32), ("num_table_shift", C.c_int32),
                ("ms", C.c_float), ("row_kernel", C.c_int32), ("sym_fill_pct", C.c_int32),
                ("num_fill_pct", C.c_int32)]


class HostCsr(C.Structure):
    """nspb_host_csr: a CSR in host memory allocated by the library."""
    _fields_ = [("nrows", C.c_int64), ("ncols", C.c_int64), ("nnz", C.c_int64),
                ("full_nrows", C.c_int64), ("first_row", C.c_int64),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


class SfCSR(C.Structure):
    """sfCSR of the reference (nsp/inc/nsp.h:57-70)."""
    _fields_ = [("rpt", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p),
                ("d_rpt", C.c_void_p), ("d_col", C.c_void_p), ("d_val", C.c_void_p),
                ("M", C.c_uint32), ("N", C.c_uint32), ("nnz", C.c_int32),
                ("nnz_max", C.c_int32), ("matrix_name", C.c_char_p)]


P = C.POINTER
_i32p = P(C.c_int32)
_f64p = P(C.c_double)

_SIGS = {
    "nspb_version": (C.c_char_p, []),
    "nspb_strerror": (C.c_char_p, [C.c_int]),
    "nspb_last_cuda_error": (C.c_int, []),
    "nspb_default_opts": (None, [P(Opts)]),
    "nspb_free": (C.c_int, [C.c_void_p]),
    "nspb_device_sm_count": (C.c_int, [P(C.c_int)]),
    "nspb_spgemm": (C.c_int, [P(CsrIn), P(CsrIn), P(CsrOut), P(Opts), P(Stats)]),
    "nspb_spgemm_symbolic": (C.c_int, [P(CsrIn), P(CsrIn), P(CsrOut), P(Opts), P(Stats)]),
    "nspb_spgemm_numeric": (C.c_int, [P(CsrIn), P(CsrIn), P(CsrOut), P(Opts), P(Stats)]),
    "nspb_intprod": (C.c_int, [P(CsrIn), P(CsrIn), C.c_void_p, P(C.c_int64), C.c_void_p]),
    "nspb_spgemm_batched": (C.c_int, [C.c_int, P(CsrIn), P(CsrIn), P(CsrOut), P(Opts), P(Stats),
                                      P(C.c_void_p), P(C.c_int32)]),
    "nspb_getmct": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p,
                              P(C.c_int64), C.c_void_p]),
    "nspb_compactcol": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p,
                                  P(C.c_int64), C.c_void_p]),
    "nspb_shrink_col": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                  C.c_void_p]),
    "nspb_spgemm_rowblocked": (C.c_int, [P(CsrIn), P(CsrIn), C.c_int64, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int64, P(C.c_int64), P(C.c_int32),
                                         P(Opts)]),
    "nspb_gen_stencil": (C.c_int64, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                     C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nspb_gen_stencil_slab": (C.c_int64, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int32, C.c_uint64, C.c_int32, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    "nspb_gen_powerlaw": (C.c_int64, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_int32,
                                      C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "nspb_gen_random": (C.c_int64, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                    C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nspb_powerlaw_xmin": (C.c_double, [C.c_double, C.c_double, C.c_int32]),
    "nspb_nsp_spgemm_kernel_hash": (C.c_int, [P(SfCSR), P(SfCSR), P(SfCSR)]),
    "nspb_plan_create": (C.c_int, [C.c_int, P(CsrIn), P(CsrIn), P(CsrOut), P(Opts), P(Stats),
                                   P(C.c_void_p)]),
    "nspb_plan_execute": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nspb_plan_destroy": (C.c_int, [C.c_void_p]),
    "nspb_autotune": (C.c_int, [P(CsrIn), P(CsrIn), P(Opts), C.c_int, P(Opts), P(TuneEntry),
                                P(C.c_int32)]),
    "nspb_spgemm_host": (C.c_int, [P(CsrIn), P(CsrIn), C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int64, P(C.c_int64), C.c_int32, P(Opts)]),
    "nspb_transpose": (C.c_int, [P(CsrIn), P(CsrOut), P(Opts)]),
    "nspb_sa_prolongator": (C.c_int, [P(CsrIn), P(CsrIn), C.c_double, P(CsrOut), P(Opts)]),
    "nspb_galerkin": (C.c_int, [P(CsrIn), P(CsrIn), P(CsrOut), P(CsrOut), P(Opts)]),
    "nspb_read_coo_bin": (C.c_int, [C.c_char_p, C.c_int, C.c_int, P(HostCsr)]),
    "nspb_read_coo_ascii": (C.c_int, [C.c_char_p, P(HostCsr)]),
    "nspb_host_csr_free": (None, [P(HostCsr)]),
    "nspb_write_coo_bin": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                     C.c_int64, C.c_int]),
    "nspb_write_mtx": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                 C.c_int64]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class NspbError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib.nspb_strerror(status).decode()
        if status == ERR_CUDA:
            msg += f" (cudaError {lib.nspb_last_cuda_error()})"
        super().__init__(f"{what}: {msg} [{status}]" if what else f"{msg} [{status}]")


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise NspbError(status, what)
