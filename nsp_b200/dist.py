"""Row-split product over several GPUs, one process per GPU: the MPI-free
counterpart of nsparseMGPU_version1 (src/spspmpi.cu:371-975).

Rank r owns rows [a_off[r], a_off[r+1]) of A (with global column ids) and
rows [p_off[r], p_off[r+1]) of P. C = A·P is formed without any reduction:

  1. the sorted unique columns of the local A rows (nspb_getmct) name the P
     rows this rank needs (get_missing_col, src/spspmpi.cu:330, called at :395);
  2. rows owned elsewhere are requested from their owners and received in
     one exchange step: all_to_all_single of the request counts, of the row
     ids, of the row lengths and of the rows' columns and values (the
     MPI_Alltoall / MPI_Alltoallv sequence of src/spspmpi.cu:495-875);
  3. the needed rows, own and received, form a compact P in ascending global
     row order ("completedP"); A's columns are remapped to positions in that
     list (nspb_shrink_col; get_shrinked_matrix, src/spspmpi.cu:166-182);
  4. the local product C_r = A_r · P_compact runs on this rank's GPU; C_r has
     P's global column ids.

The exchange moves tensors with torch.distributed (NCCL on GPUs; gloo for
CPU tensors). Its bookkeeping (owners, splits, gathers) is plain tensor
indexing on whatever device the tensors live on, so it runs unchanged under
gloo on the CPU; steps 1, 3 and 4 call this library's kernels and need a GPU.
"""
from __future__ import annotations

import ctypes as C

from ._lib import check, lib
from .csr import DeviceCSR


def row_offsets(n: int, world: int) -> list[int]:
    """The reference's row split (src/READ_MATRIX_MPI.cpp:257-258): n // world
    rows per rank, the last rank also takes the remainder."""
    per = n // world
    return [r * per for r in range(world)] + [n]


def balanced_offsets(row_work, world: int) -> list[int]:
    """Contiguous row blocks balanced by work: block r ends at the first row
    where the prefix sum of `row_work` (the intermediate products of each row
    of A, nspb_intprod) reaches (r+1)/world of the total. The reference splits
    by row count (src/READ_MATRIX_MPI.cpp:256-270), which leaves the rank that
    owns a power-law matrix's hub rows with most of the product. No block is
    heavier than the ideal share plus the heaviest single row. Every rank
    derives the same offsets from the same weights."""
    import numpy as np
    w = np.asarray(row_work, dtype=np.float64).ravel()
    n = w.size
    pre = np.concatenate(([0.0], np.cumsum(w)))
    total = pre[-1]
    if world <= 1 or n == 0 or total <= 0.0:
        return row_offsets(n, max(world, 1))
    targets = total * np.arange(1, world) / world
    cuts = np.searchsorted(pre, targets, side="left")  # first prefix >= target
    cuts = np.clip(cuts, 0, n)
    return [0] + [int(c) for c in np.maximum.accumulate(cuts)] + [n]


def _a2a(out, inp, out_splits, in_splits, group):
    import torch.distributed as dist
    dist.all_to_all_single(out, inp, out_splits, in_splits, group=group)


def _ranges(starts, lens):
    """Concatenation of the index ranges [starts[i], starts[i] + lens[i])."""
    import torch
    if lens.numel() == 0:
        return torch.zeros(0, dtype=torch.int64, device=lens.device)
    excl = torch.cumsum(lens, 0) - lens
    return (torch.repeat_interleave(starts - excl, lens)
            + torch.arange(int(lens.sum()), device=lens.device))


def exchange_rows(rowptr, col, val, p_off, rank: int, needed, group=None):
    """The rows `needed` (sorted unique global row ids, any owners) of a
    row-partitioned P, in that order, as (rowptr int32, col, val) tensors on
    the device of `col`. rowptr/col/val hold this rank's rows [p_off[rank],
    p_off[rank+1]) of P. Every rank of `group` calls this together; a rank
    sends only rows that another rank asked for."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = col.device
    lo = p_off[rank]
    rp = rowptr.to(torch.int64)
    need = needed.to(torch.int64)
    owner = torch.searchsorted(torch.tensor(p_off[1:], dtype=torch.int64, device=dev), need,
                               right=True)
    remote = owner != rank
    req = need[remote]  # ascending, hence grouped by owner in rank order
    send_cnt = torch.bincount(owner[remote], minlength=world).to(torch.int64)
    recv_cnt = torch.empty_like(send_cnt)
    dist.all_to_all_single(recv_cnt, send_cnt, group=group)
    sc, rc = send_cnt.tolist(), recv_cnt.tolist()
    asked = torch.empty(sum(rc), dtype=torch.int64, device=dev)  # rows others want from me
    _a2a(asked, req, rc, sc, group)
    aloc = asked - lo
    alen = rp[aloc + 1] - rp[aloc]
    glen = torch.empty(sum(sc), dtype=torch.int64, device=dev)  # lengths of the rows I asked for
    _a2a(glen, alen, sc, rc, group)
    send_tot = [int(t.sum()) for t in torch.split(alen, rc)]
    recv_tot = [int(t.sum()) for t in torch.split(glen, sc)]
    pidx = _ranges(rp[aloc], alen)
    rcol = torch.empty(sum(recv_tot), dtype=col.dtype, device=dev)
    rval = torch.empty(sum(recv_tot), dtype=val.dtype, device=dev)
    _a2a(rcol, col[pidx], recv_tot, send_tot, group)
    _a2a(rval, val[pidx], recv_tot, send_tot, group)
    # own rows from the local arrays, received rows in arrival order (by owner
    # rank, then request order: ascending, like `need`)
    own = ~remote
    oloc = need[own] - lo
    nlen = torch.empty(need.numel(), dtype=torch.int64, device=dev)
    nlen[own] = rp[oloc + 1] - rp[oloc]
    nlen[remote] = glen
    out_rp = torch.zeros(need.numel() + 1, dtype=torch.int64, device=dev)
    torch.cumsum(nlen, 0, out=out_rp[1:])
    total = int(out_rp[-1])
    out_col = torch.empty(total, dtype=col.dtype, device=dev)
    out_val = torch.empty(total, dtype=val.dtype, device=dev)
    dst_own = _ranges(out_rp[:-1][own], nlen[own])
    src_own = _ranges(rp[oloc], nlen[own])
    out_col[dst_own] = col[src_own]
    out_val[dst_own] = val[src_own]
    dst_rem = _ranges(out_rp[:-1][remote], nlen[remote])
    out_col[dst_rem] = rcol
    out_val[dst_rem] = rval
    return out_rp.to(torch.int32), out_col, out_val


def _getmct_all(col):
    """Sorted unique values of col (nspb_getmct with first > last)."""
    import torch
    n = col.numel()
    out = torch.empty(max(n, 1), dtype=torch.int32, device=col.device)
    cnt = C.c_int64(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.nspb_getmct(C.c_void_p(col.data_ptr()), n, 1, 0, C.c_void_p(out.data_ptr()),
                          C.byref(cnt), stream), "nspb_getmct")
    return out[:cnt.value]


def _shrink(col, cols):
    import torch
    out = torch.empty(max(col.numel(), 1), dtype=torch.int32, device=col.device)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.nspb_shrink_col(C.c_void_p(col.data_ptr()), col.numel(),
                              C.c_void_p(cols.data_ptr()), cols.numel(),
                              C.c_void_p(out.data_ptr()), stream), "nspb_shrink_col")
    return out[:col.numel()]


def halo_product(A_local: DeviceCSR, P_local: DeviceCSR, p_off: list[int], rank: int,
                 group=None, **spgemm_kw) -> DeviceCSR:
    """C_r = A_r · P for this rank's rows of A (steps 1-4 above)."""
    from . import spgemm
    needed = _getmct_all(A_local.col)
    rp, col, val = exchange_rows(P_local.rowptr, P_local.col, P_local.val, p_off, rank,
                                 needed, group)
    Pc = DeviceCSR(needed.numel(), P_local.ncols, rp, col, val)
    Ac = DeviceCSR(A_local.nrows, needed.numel(), A_local.rowptr, _shrink(A_local.col, needed),
                   A_local.val)
    return spgemm(Ac, Pc, **spgemm_kw)
