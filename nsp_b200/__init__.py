"""nsp_b200 — B200-native (sm_100a) CSR sparse matrix product C = A·B.

The product runs in libnspb.so (hand-written CUDA kernels behind the C ABI
of include/nspb.h). This package is the Python glue used by the tests and
the benchmark: ctypes bindings, CSR containers and the seeded generators.

Entry points mirroring the reference (amavliut/nsp):
  nsp_spgemm_kernel_hash(a, b, c)   nsp/inc/nsp.h:105 on sfCSR structs
  nsparseMGPU_version1(A, B)        src/spspmpi.h:31 (one GPU) -> (C, loc_time)
  spgemm(A, B, ...)                 the C-ABI one-call product
"""
from __future__ import annotations

import ctypes as C
import os

from . import gen, matio
from ._lib import (F32, F64, PREC_FP32_COMP, PREC_FP32_WIDE, PREC_FP64, CsrIn, CsrOut, NspbError, Opts,
                   SfCSR, Stats, check, lib)
from .csr import DeviceCSR, HostCSR, adopt

__all__ = ["spgemm", "spgemm_symbolic", "spgemm_numeric", "intprod", "nsp_spgemm_kernel_hash",
           "nsparseMGPU_version1", "DeviceCSR", "HostCSR", "gen", "NspbError", "lib",
           "make_opts", "stats_dict", "matio", "transpose", "sa_prolongator", "galerkin", "Plan",
           "autotune", "spgemm_host"]


def _stream_ptr(stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _precision(name: str) -> int:
    """"fp64", "fp32c" (fp32 pairs, two-sum compensated) or "fp32w" (fp32
    inputs, fp64 accumulation of exact products)."""
    return {"fp64": PREC_FP64, "fp32c": PREC_FP32_COMP, "fp32w": PREC_FP32_WIDE}[precision_name(name)]


def precision_name(name: str) -> str:
    if name not in ("fp64", "fp32c", "fp32w"):
        raise ValueError(f"precision {name!r}: expected fp64, fp32c or fp32w")
    return name


def make_opts(precision=PREC_FP64, assume_sorted=False, check_errors=True, group_lanes=0,
              comp_tol=1e-10, stream=None, table_shift=0, row_kernel=None) -> Opts:
    """nspb_opts for the Python entry points. row_kernel None takes
    NSPB_ROW_KERNEL from the environment (0 when unset): the test suite runs
    once per row-group kernel family that way."""
    if row_kernel is None:
        row_kernel = int(os.environ.get("NSPB_ROW_KERNEL", "0"), 0)
    o = Opts()
    lib.nspb_default_opts(C.byref(o))
    o.precision = precision
    o.assume_sorted = int(assume_sorted)
    o.check_errors = int(check_errors)
    o.group_lanes = int(group_lanes)
    o.comp_tol = float(comp_tol)
    o.stream = _stream_ptr(stream)
    o.num_table_shift = int(table_shift)
    o.row_kernel = int(row_kernel)
    return o


def stats_dict(s: Stats) -> dict:
    return {"intprod": s.intprod, "nnz": s.nnz, "sym_bins": list(s.sym_bins)[:12],
            "num_bins": list(s.num_bins)[:10], "rows_redone": s.rows_redone,
            "b_sorted": s.b_sorted, "max_row_err": s.max_row_err, "launches": s.launches,
            "entry_map": s.entry_map}


def spgemm(A: DeviceCSR, B: DeviceCSR, precision: str = "fp64", out: DeviceCSR | None = None,
           stream=None, check_errors: bool = True, assume_sorted: bool = False,
           group_lanes: int = 0, comp_tol: float = 1e-10, return_stats: bool = False,
           table_shift: int = 0, row_kernel: int | None = None, sym_fill_pct: int = 0,
           num_fill_pct: int = 0):
    """C = A·B on the current CUDA device through nspb_spgemm.

    With `out` given, its tensors are used as C's arrays (capacity = their
    length); otherwise the library allocates C (freed with the tensors)."""
    import torch
    prec = _precision(precision)
    o = make_opts(prec, assume_sorted, check_errors, group_lanes, comp_tol, stream, table_shift,
                  row_kernel)
    o.sym_fill_pct, o.num_fill_pct = int(sym_fill_pct), int(num_fill_pct)
    a, b = A.as_in(), B.as_in()
    c = CsrOut()
    if out is not None:
        c.rowptr = out.rowptr.data_ptr()
        c.col = out.col.data_ptr()
        c.val = out.val.data_ptr()
        c.capacity = min(out.col.numel(), out.val.numel())
    st = Stats()
    check(lib.nspb_spgemm(C.byref(a), C.byref(b), C.byref(c), C.byref(o), C.byref(st)),
          "nspb_spgemm")
    if out is not None:
        res = DeviceCSR(A.nrows, B.ncols, out.rowptr, out.col[:c.nnz], out.val[:c.nnz])
    else:
        res = DeviceCSR(A.nrows, B.ncols, adopt(c.rowptr, A.nrows + 1, "int32"),
                        adopt(c.col, c.nnz, "int32"), adopt(c.val, c.nnz, "float64"))
    return (res, stats_dict(st)) if return_stats else res


def _adopt_out(c: CsrOut, vdtype="float64") -> DeviceCSR:
    return DeviceCSR(c.nrows, c.ncols, adopt(c.rowptr, c.nrows + 1, "int32"),
                     adopt(c.col, c.nnz, "int32"), adopt(c.val, c.nnz, vdtype))


def transpose(A: DeviceCSR, stream=None) -> DeviceCSR:
    """A^T through nspb_transpose (rows of the result list A's rows ascending;
    the reference's CSRm::T, src/CSR.cu:738-785)."""
    import torch
    o = make_opts(stream=stream)
    a, t = A.as_in(), CsrOut()
    check(lib.nspb_transpose(C.byref(a), C.byref(t), C.byref(o)), "nspb_transpose")
    return _adopt_out(t, "float32" if A.val.dtype == torch.float32 else "float64")


def sa_prolongator(A: DeviceCSR, Ptent: DeviceCSR, omega: float = 2.0 / 3.0,
                   stream=None) -> DeviceCSR:
    """P = P_tent - omega D^-1 (A P_tent) through nspb_sa_prolongator."""
    o = make_opts(stream=stream)
    a, t, p = A.as_in(), Ptent.as_in(), CsrOut()
    check(lib.nspb_sa_prolongator(C.byref(a), C.byref(t), C.c_double(omega), C.byref(p),
                                  C.byref(o)), "nspb_sa_prolongator")
    return _adopt_out(p)


def galerkin(A: DeviceCSR, P: DeviceCSR, return_R: bool = False, stream=None):
    """A_c = R (A P) with R = P^T through nspb_galerkin; (A_c, R) with return_R."""
    o = make_opts(stream=stream)
    a, p, r, ac = A.as_in(), P.as_in(), CsrOut(), CsrOut()
    check(lib.nspb_galerkin(C.byref(a), C.byref(p), C.byref(r) if return_R else None,
                            C.byref(ac), C.byref(o)), "nspb_galerkin")
    Ac = _adopt_out(ac)
    return (Ac, _adopt_out(r)) if return_R else Ac


def autotune(A: DeviceCSR, B: DeviceCSR, precision: str = "fp64", reps: int = 3, stream=None):
    """nspb_autotune: (knobs of the fastest candidate, [(knobs, ms), ...] for
    every candidate timed). knobs: group_lanes, table_shift, row_kernel,
    sym_fill_pct, num_fill_pct."""
    from ._lib import TuneEntry
    o = make_opts(_precision(precision), stream=stream)
    best = Opts()
    rep = (TuneEntry * 16)()
    n = C.c_int32(0)
    a, b = A.as_in(), B.as_in()
    check(lib.nspb_autotune(C.byref(a), C.byref(b), C.byref(o), int(reps), C.byref(best), rep,
                            C.byref(n)), "nspb_autotune")

    def knobs(x):
        return {"group_lanes": x.group_lanes, "table_shift": x.num_table_shift,
                "row_kernel": x.row_kernel, "sym_fill_pct": x.sym_fill_pct,
                "num_fill_pct": x.num_fill_pct}
    return knobs(best), [(knobs(rep[i]), rep[i].ms) for i in range(n.value)]


def _host_ptr(x):
    import numpy as np
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()  # CPU (pinned) torch tensor


def spgemm_host(A, B, out=None, nblocks: int = 0, precision: str = "fp64", stream=None):
    """C = A·B with host operands through nspb_spgemm_host. A and B expose
    nrows, ncols and host arrays rowptr/col/val (numpy, or CPU torch tensors,
    pinned for overlapped copies). With `out` = (rowptr, col, val) host arrays
    of enough capacity C is written there; otherwise numpy arrays are sized by
    a first call. Returns (rowptr, col, val)."""
    import numpy as np
    prec = _precision(precision)
    o = make_opts(prec, stream=stream)

    def host_in(M):
        d = CsrIn()
        d.nrows, d.ncols = M.nrows, M.ncols
        d.nnz = int(M.rowptr[M.nrows])
        d.rowptr, d.col, d.val = _host_ptr(M.rowptr), _host_ptr(M.col), _host_ptr(M.val)
        d.val_type = F32 if str(M.val.dtype).endswith("float32") else F64
        return d
    a, b = host_in(A), host_in(B)
    nnz = C.c_int64(0)
    if out is None:
        rp = np.empty(A.nrows + 1, np.int32)
        st = lib.nspb_spgemm_host(C.byref(a), C.byref(b), rp.ctypes.data, None, None, 0,
                                  C.byref(nnz), int(nblocks), C.byref(o))
        if st not in (0, -8):
            check(st, "nspb_spgemm_host")
        out = (rp, np.empty(max(nnz.value, 1), np.int32), np.empty(max(nnz.value, 1), np.float64))
    rp, col, val = out
    cap = min(len(col), len(val))
    check(lib.nspb_spgemm_host(C.byref(a), C.byref(b), _host_ptr(rp), _host_ptr(col), _host_ptr(val),
                               cap, C.byref(nnz), int(nblocks), C.byref(o)), "nspb_spgemm_host")
    return rp, col[:nnz.value], val[:nnz.value]


class _PlanView:
    """Non-owning view of a plan-owned device array; keeps the plan alive."""

    def __init__(self, plan, ptr: int, count: int, typestr: str):
        self.plan, self.ptr, self.count, self.typestr = plan, int(ptr or 0), int(count), typestr

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.count,), "typestr": self.typestr,
                "data": (self.ptr, False), "version": 2, "strides": None}


class Plan:
    """Products of a fixed structure formed again and again (nspb_plan_*):
    the symbolic phase and C's allocation happen once, execute() replays the
    numeric phase from a CUDA graph with the current values of the inputs.
    `C[p]` are DeviceCSR views of the plan's arrays."""

    def __init__(self, As, Bs, precision: str = "fp64", check_errors: bool = True, stream=None,
                 max_group: int = 0):
        import torch
        m = len(As)
        prec = _precision(precision)
        o = make_opts(prec, False, check_errors, 0, 1e-10, stream)
        o.batch_max_products = int(max_group)
        a = (CsrIn * m)(*[x.as_in() for x in As])
        b = (CsrIn * m)(*[x.as_in() for x in Bs])
        c = (CsrOut * m)()
        st = Stats()
        h = C.c_void_p()
        check(lib.nspb_plan_create(m, a, b, c, C.byref(o), C.byref(st), C.byref(h)),
              "nspb_plan_create")
        self._h = h
        self._inputs = (list(As), list(Bs))  # the graph reads their arrays
        self.stats = stats_dict(st)

        def view(ptr, cnt, ts, dt):
            if cnt == 0:  # an empty product's pointer may sit one past an allocation
                return torch.empty(0, dtype=dt, device="cuda")
            return torch.as_tensor(_PlanView(self, ptr, cnt, ts), device="cuda").view(dt)
        self.C = [DeviceCSR(c[p].nrows, c[p].ncols, view(c[p].rowptr, c[p].nrows + 1, "<i4", torch.int32),
                            view(c[p].col, c[p].nnz, "<i4", torch.int32),
                            view(c[p].val, c[p].nnz, "<f8", torch.float64)) for p in range(m)]

    def execute(self, stream=None) -> None:
        check(lib.nspb_plan_execute(self._h, _stream_ptr(stream)), "nspb_plan_execute")

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.nspb_plan_destroy(self._h)
            self._h = C.c_void_p()


def spgemm_batched(As, Bs, precision: str = "fp64", stream=None, return_stats: bool = False,
                   max_group: int = 0):
    """C[p] = A[p]·B[p] for every pair through nspb_spgemm_batched (one
    block-diagonal product per group of products). Returns DeviceCSRs whose
    tensors view the shared output allocations (freed with the last view)."""
    import torch
    m = len(As)
    prec = _precision(precision)
    o = make_opts(prec, False, True, 0, 1e-10, stream)
    o.batch_max_products = int(max_group)
    a = (CsrIn * m)(*[x.as_in() for x in As])
    b = (CsrIn * m)(*[x.as_in() for x in Bs])
    c = (CsrOut * m)()
    owners = (C.c_void_p * (3 * m + 3))()
    n_own = C.c_int32(0)
    st = Stats()
    check(lib.nspb_spgemm_batched(m, a, b, c, C.byref(o), C.byref(st), owners, C.byref(n_own)),
          "nspb_spgemm_batched")
    # one tensor per owner allocation; each product's arrays are slices of them
    from .csr import DevBuf
    bases = {}
    for q in range(n_own.value):
        bases[owners[q]] = None
    ptrs = sorted(bases)
    out = []

    def owner_of(ptr):
        lo = max(p_ for p_ in ptrs if p_ <= ptr)
        return lo

    views = {}
    sizes = {}
    for p in range(m):
        for ptr, cnt, es in ((c[p].rowptr, c[p].nrows + 1, 4), (c[p].col, c[p].nnz, 4),
                             (c[p].val, c[p].nnz, 8)):
            base = owner_of(ptr)
            sizes[base] = max(sizes.get(base, 0), ptr - base + cnt * es)
    for base, nbytes in sizes.items():
        views[base] = torch.as_tensor(DevBuf(base, nbytes, "|u1"), device="cuda")
    for p in range(m):
        def sl(ptr, cnt, dtype):
            base = owner_of(ptr)
            raw = views[base][ptr - base: ptr - base + cnt * torch.empty((), dtype=dtype).element_size()]
            return raw.view(dtype)
        out.append(DeviceCSR(c[p].nrows, c[p].ncols, sl(c[p].rowptr, c[p].nrows + 1, torch.int32),
                             sl(c[p].col, c[p].nnz, torch.int32),
                             sl(c[p].val, c[p].nnz, torch.float64)))
    return (out, stats_dict(st)) if return_stats else out


def spgemm_symbolic(A: DeviceCSR, B: DeviceCSR, stream=None, assume_sorted=False):
    """Two-call form, step 1: returns (rowptr tensor, nnz)."""
    import torch
    o = make_opts(PREC_FP64, assume_sorted, True, 0, 1e-12, stream)
    if A.val.dtype == torch.float32:
        o.precision = PREC_FP32_COMP
    a, b = A.as_in(), B.as_in()
    rowptr = torch.empty(A.nrows + 1, dtype=torch.int32, device=A.rowptr.device)
    c = CsrOut()
    c.rowptr = rowptr.data_ptr()
    check(lib.nspb_spgemm_symbolic(C.byref(a), C.byref(b), C.byref(c), C.byref(o), None),
          "nspb_spgemm_symbolic")
    return rowptr, int(c.nnz)


def spgemm_numeric(A: DeviceCSR, B: DeviceCSR, rowptr, nnz: int, precision="fp64",
                   stream=None, assume_sorted=False) -> DeviceCSR:
    """Two-call form, step 2: fills col/val for the given rowptr."""
    import torch
    prec = _precision(precision)
    o = make_opts(prec, assume_sorted, True, 0, 1e-12, stream)
    a, b = A.as_in(), B.as_in()
    col = torch.empty(max(nnz, 1), dtype=torch.int32, device=rowptr.device)
    val = torch.empty(max(nnz, 1), dtype=torch.float64, device=rowptr.device)
    c = CsrOut()
    c.nnz = nnz
    c.rowptr = rowptr.data_ptr()
    c.col = col.data_ptr()
    c.val = val.data_ptr()
    c.capacity = max(nnz, 1)
    check(lib.nspb_spgemm_numeric(C.byref(a), C.byref(b), C.byref(c), C.byref(o), None),
          "nspb_spgemm_numeric")
    return DeviceCSR(A.nrows, B.ncols, rowptr, col[:nnz], val[:nnz])


def intprod(A: DeviceCSR, B: DeviceCSR, stream=None):
    """Per-row intermediate-product counts (int64 tensor) and their total."""
    import torch
    row_ip = torch.empty(max(A.nrows, 1), dtype=torch.int64, device=A.rowptr.device)
    tot = C.c_int64(0)
    a, b = A.as_in(), B.as_in()
    check(lib.nspb_intprod(C.byref(a), C.byref(b), C.c_void_p(row_ip.data_ptr()),
                           C.byref(tot), _stream_ptr(stream)), "nspb_intprod")
    return row_ip[:A.nrows], int(tot.value)


def sfcsr_of(m: DeviceCSR) -> SfCSR:
    """sfCSR view of a device CSR (nsp/inc/nsp.h:57-70)."""
    s = SfCSR()
    s.M = m.nrows
    s.N = m.ncols
    s.nnz = m.nnz
    s.d_rpt = m.rowptr.data_ptr()
    s.d_col = m.col.data_ptr() if m.nnz else None
    s.d_val = m.val.data_ptr() if m.nnz else None
    return s


def nsp_spgemm_kernel_hash(a: SfCSR, b: SfCSR, c: SfCSR) -> None:
    """The reference entry point (nsp/inc/nsp.h:105): fills c->M, N, nnz and
    cudaMalloc'ed c->d_rpt/d_col/d_val. Raises NspbError on failure (the C++
    shim of the same name exits the process instead, like the reference)."""
    check(lib.nspb_nsp_spgemm_kernel_hash(C.byref(a), C.byref(b), C.byref(c)),
          "nsp_spgemm_kernel_hash")


def nsparseMGPU_version1(A: DeviceCSR, B: DeviceCSR):
    """One-GPU nsparseMGPU_version1 (src/spspmpi.cu:371, nprocs == 1 path):
    returns (C, loc_time) with loc_time the wall seconds of the product
    bracketed by device synchronisation (src/spspmpi.cu:288-305)."""
    import time
    import torch
    a, b, c = sfcsr_of(A), sfcsr_of(B), SfCSR()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nsp_spgemm_kernel_hash(a, b, c)
    torch.cuda.synchronize()
    loc = time.perf_counter() - t0
    res = DeviceCSR(c.M, c.N, adopt(c.d_rpt, c.M + 1, "int32"), adopt(c.d_col, c.nnz, "int32"),
                    adopt(c.d_val, c.nnz, "float64"))
    return res, loc


def spgemm_rowblocked(A: DeviceCSR, B: DeviceCSR, budget_bytes: int, stream=None):
    """C = A·B computed in row blocks whose C fits `budget_bytes` of device
    memory, written to host arrays; returns (HostCSR, number of blocks)."""
    import numpy as np
    from .csr import HostCSR
    a, b = A.as_in(), B.as_in()
    o = make_opts(PREC_FP64, False, True, 0, 1e-10, stream)
    rp = np.empty(A.nrows + 1, dtype=np.int32)
    nnz = C.c_int64(0)
    nblk = C.c_int32(0)
    # size pass: capacity 0 reports nnz(C) through NSPB_ERR_CAPACITY
    st = lib.nspb_spgemm_rowblocked(C.byref(a), C.byref(b), int(budget_bytes),
                                    rp.ctypes.data, None, None, 0, C.byref(nnz),
                                    C.byref(nblk), C.byref(o))
    if st not in (0, -8):
        check(st, "nspb_spgemm_rowblocked")
    col = np.empty(max(nnz.value, 1), dtype=np.int32)
    val = np.empty(max(nnz.value, 1), dtype=np.float64)
    check(lib.nspb_spgemm_rowblocked(C.byref(a), C.byref(b), int(budget_bytes), rp.ctypes.data,
                                     col.ctypes.data, val.ctypes.data, nnz.value, C.byref(nnz),
                                     C.byref(nblk), C.byref(o)), "nspb_spgemm_rowblocked")
    n = nnz.value
    return HostCSR(A.nrows, B.ncols, rp, col[:n], val[:n]), int(nblk.value)
