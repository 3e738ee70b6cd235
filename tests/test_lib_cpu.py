"""The C-ABI library loads and exports every symbol its headers declare
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

import nsp_b200 as nb
from nsp_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_c_functions():
    names = set()
    for h in ("nspb.h", "nspb_compat.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(nspb_\w+)\s*\(", src))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_c_functions()
    assert "nspb_spgemm" in names and "nspb_nsp_spgemm_kernel_hash" in names
    assert len(names) >= 20


@pytest.mark.parametrize("name", declared_c_functions())
def test_c_symbol_exported(name):
    assert hasattr(_lib.lib, name), f"{name} missing from libnspb.so"


def test_cpp_shims_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for sym in ("_Z22nsp_spgemm_kernel_hashP5sfCSRS0_S0_",
                "nsparseMGPU_version0", "nsparseMGPU_version1"):
        assert sym in out, sym


def test_strerror_and_defaults():
    assert nb.lib.nspb_strerror(0) == b"success"
    assert b"int32" in nb.lib.nspb_strerror(_lib.ERR_OVERFLOW)
    o = _lib.Opts()
    nb.lib.nspb_default_opts(ctypes.byref(o))
    assert o.precision == _lib.PREC_FP64 and o.comp_tol == 1e-10


def test_generator_thread_independent():
    code = ("import nsp_b200 as nb, hashlib; P = nb.gen.powerlaw(20000, max_deg=2000, seed=3);"
            "print(hashlib.sha1(P.col.tobytes() + P.val.tobytes()).hexdigest())")
    outs = set()
    for th in ("1", "4"):
        env = dict(os.environ, OMP_NUM_THREADS=th)
        outs.add(subprocess.run(["python", "-c", code], cwd=ROOT, env=env, capture_output=True,
                                text=True, check=True).stdout.strip())
    assert len(outs) == 1


def test_no_device_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    a = _lib.CsrIn()
    c = _lib.CsrOut()
    st = nb.lib.nspb_spgemm(ctypes.byref(a), ctypes.byref(a), ctypes.byref(c), None, None)
    assert st == _lib.ERR_NO_DEVICE


def test_header_is_plain_c_and_layouts_match(tmp_path):
    """include/nspb.h compiles as C99 with warnings as errors, a C program
    links libnspb.so, and the struct sizes it sees equal the Python
    bindings' (no GPU call is made)."""
    src = tmp_path / "abi.c"
    src.write_text(r'''
#include <stdio.h>
#include "nspb.h"
int main(void) {
  nspb_opts o;
  nspb_default_opts(&o);
  printf("%zu %zu %zu %zu %zu %zu %zu %d %s\n", sizeof(nspb_csr_in), sizeof(nspb_csr_out),
         sizeof(nspb_opts), sizeof(nspb_stats), sizeof(nspb_host_csr), sizeof(nspb_tune_entry),
         sizeof(void *), o.precision, nspb_version());
  return o.comp_tol > 0.0 ? 0 : 1;
}
''')
    exe = tmp_path / "abi"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["/usr/bin/gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lnspb", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(x) for x in out[:7]]
    assert sizes == [ctypes.sizeof(_lib.CsrIn), ctypes.sizeof(_lib.CsrOut),
                     ctypes.sizeof(_lib.Opts), ctypes.sizeof(_lib.Stats),
                     ctypes.sizeof(_lib.HostCsr), ctypes.sizeof(_lib.TuneEntry), 8]
    assert int(out[7]) == _lib.PREC_FP64


def _host_in(M, val_type=_lib.F64):
    d = _lib.CsrIn()
    d.nrows, d.ncols, d.nnz = M.nrows, M.ncols, int(M.rowptr[M.nrows])
    d.rowptr, d.col, d.val = M.rowptr.ctypes.data, M.col.ctypes.data, M.val.ctypes.data
    d.val_type = val_type
    return d


def test_host_entry_checks_arguments_before_the_device():
    """nspb_spgemm_host rejects malformed host operands with
    NSPB_ERR_INVALID before any CUDA call, so the same statuses come back with
    or without a GPU."""
    import numpy as np
    A = nb.gen.random(50, 40, 1, 5, seed=1)
    B = nb.gen.random(40, 30, 1, 5, seed=2)
    rp = np.empty(A.nrows + 1, np.int32)
    nnz = ctypes.c_int64(0)

    def call(a, b, nnz_out=ctypes.byref(nnz), rowptr=rp.ctypes.data):
        return nb.lib.nspb_spgemm_host(ctypes.byref(a), ctypes.byref(b), rowptr, None, None, 0,
                                       nnz_out, 0, None)

    a, b = _host_in(A), _host_in(B)
    assert call(a, _host_in(B, val_type=_lib.F32)) == _lib.ERR_INVALID  # value types differ
    assert call(_host_in(B), b) == _lib.ERR_INVALID                      # ncols(A) != nrows(B)
    assert call(a, b, nnz_out=None) == _lib.ERR_INVALID
    assert call(a, b, rowptr=None) == _lib.ERR_INVALID
    bad = _host_in(A)
    bad.nnz = A.nnz - 1                                                   # rowptr[n] != nnz
    assert call(bad, b) == _lib.ERR_INVALID
    shifted = A.rowptr + 1                                                # rowptr[0] != 0
    s = _host_in(A)
    s.rowptr = shifted.ctypes.data
    assert call(s, b) == _lib.ERR_INVALID
    import torch
    if not torch.cuda.is_available():
        assert call(a, b) == _lib.ERR_NO_DEVICE
