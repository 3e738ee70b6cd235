"""Time the reference's own nsp_spgemm_kernel_hash (built for sm_100a from
the reference sources into oracle/_ref/libnsp_ref.so) against this
library's drop-in of the same entry point, on the same device inputs.

Both calls allocate C inside with cudaMalloc (the reference's contract), so
the two figures compare like with like; the library's preallocated-output
figure is bench.py's `value`. Needs a GPU. Run from the repository root:

    python tests/ref_timing.py --grid 128 --reps 5

Inputs are checked on the CPU first so the reference never reaches its
unbounded chunk kernel (see tests/golden/make_golden.py).
"""
import argparse
import ctypes as C
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import torch  # noqa: E402

import nsp_b200 as nb  # noqa: E402
import oracle  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warm", type=int, default=2)
    args = ap.parse_args()
    A = nb.gen.stencil(args.grid, npts=27)
    ip, tot = oracle.intprod(A, A)
    # 27-point stencil squared: <= 125 entries per row, far from the
    # reference's chunk bin (> 3584 entries); its largest symbolic bin is 4
    assert ip.max() <= 729 and ip.max() > 512
    dA = A.to_device()
    lib = C.CDLL(oracle.REF_SO)
    lib.ref_nsp_time_device.restype = C.c_float
    lib.ref_nsp_time_device.argtypes = [C.c_int] * 3 + [C.c_void_p] * 3 + [C.c_int] + \
        [C.c_void_p] * 3 + [C.c_int] * 3 + [C.POINTER(C.c_int)]
    nnz = C.c_int(0)
    p = (dA.rowptr.data_ptr(), dA.col.data_ptr(), dA.val.data_ptr())
    ref_ms = lib.ref_nsp_time_device(A.nrows, A.ncols, A.ncols, *p, A.nnz, *p, A.nnz,
                                     args.warm, args.reps, C.byref(nnz))
    torch.cuda.synchronize()
    # this library's drop-in, same contract (C cudaMalloc'ed inside each call)
    a = nb.sfcsr_of(dA)
    times = []
    for r in range(args.warm + args.reps):
        c = nb.SfCSR()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        nb.nsp_spgemm_kernel_hash(a, a, c)
        e1.record()
        torch.cuda.synchronize()
        if r >= args.warm:
            times.append(e0.elapsed_time(e1))
        assert c.nnz == nnz.value
        for ptr in (c.d_rpt, c.d_col, c.d_val):
            nb.lib.nspb_free(C.c_void_p(ptr))
    ours = sum(times) / len(times)
    flops = 2.0 * tot
    print(json.dumps({"workload": f"stencil27_{args.grid}^3_AxA_fp64", "nnz_c": nnz.value,
                      "reference_nsp_ms": ref_ms, "reference_nsp_gflops": flops / ref_ms / 1e6,
                      "nspb_dropin_ms": ours, "nspb_dropin_gflops": flops / ours / 1e6,
                      "speedup": ref_ms / ours, "reps": args.reps}))


if __name__ == "__main__":
    main()
