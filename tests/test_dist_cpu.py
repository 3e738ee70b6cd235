"""Row-split product across ranks (nsp_b200.dist), on the CPU with gloo.

Each rank owns a block of A's rows and of P's rows (the reference's split);
exchange_rows gathers the P rows its A block references from their owners in
one all_to_all exchange. The test checks the assembled rows against the
global P, then forms the rank's block of C with the oracle over the compact
P and compares it with the oracle's global product, row block by row block.
The GPU steps of dist.halo_product (getmct, shrink_col, the product) are
covered by the GPU tests; here the same steps are restated with numpy.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import nsp_b200 as nb
import oracle
from nsp_b200 import dist as nd
from nsp_b200.csr import HostCSR


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(n, m, seed):
    A = nb.gen.random(n, n, 0, 12, seed=seed)
    P = nb.gen.random(n, m, 0, 7, seed=seed + 1)
    return A, P


def _rank_main(rank, world, port, n, m, seed, out_dir, balanced=False):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        A, P = _problem(n, m, seed)
        off = nd.row_offsets(n, world)  # P keeps the reference's split
        # A's rows: the same split, or blocks balanced by intermediate products
        a_off = nd.balanced_offsets(oracle.intprod(A, P)[0], world) if balanced else off
        r0, r1 = a_off[rank], a_off[rank + 1]
        Al, Pl = A.row_block(r0, r1), P.row_block(off[rank], off[rank + 1])
        needed = np.unique(Al.col).astype(np.int32)
        rp, col, val = nd.exchange_rows(torch.from_numpy(Pl.rowptr), torch.from_numpy(Pl.col),
                                        torch.from_numpy(Pl.val), off, rank,
                                        torch.from_numpy(needed))
        rp, col, val = rp.numpy(), col.numpy(), val.numpy()
        # the assembled rows are P's rows `needed`, in order
        for q, g in enumerate(needed):
            a, b = P.rowptr[g], P.rowptr[g + 1]
            assert np.array_equal(col[rp[q]:rp[q + 1]], P.col[a:b])
            assert np.array_equal(val[rp[q]:rp[q + 1]], P.val[a:b])
        Pc = HostCSR(len(needed), m, rp, col, val)
        Ac = HostCSR(Al.nrows, len(needed), Al.rowptr,
                     np.searchsorted(needed, Al.col).astype(np.int32), Al.val)
        crp, ccol, cval = oracle.spgemm(Ac, Pc)
        grp, gcol, gval = oracle.spgemm(A, P)
        lo, hi = grp[r0], grp[r1]
        assert np.array_equal(crp, grp[r0:r1 + 1] - lo)
        assert np.array_equal(ccol, gcol[lo:hi])
        assert np.array_equal(cval, gval[lo:hi])
        open(os.path.join(out_dir, f"ok{rank}"), "w").close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_row_split(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, _free_port(), 2500, 1800, 17, str(tmp_path)),
                       nprocs=world, start_method="spawn", join=True)
    assert sorted(os.listdir(tmp_path)) == [f"ok{r}" for r in range(world)]


def test_halo_exchange_intprod_balanced_split(tmp_path):
    """A split by the prefix of intermediate products while P keeps the
    reference's split: rows of A and P then have different owners."""
    import torch.multiprocessing as mp
    world = 3
    mp.start_processes(_rank_main, args=(world, _free_port(), 2500, 1800, 23, str(tmp_path), True),
                       nprocs=world, start_method="spawn", join=True)
    assert sorted(os.listdir(tmp_path)) == [f"ok{r}" for r in range(world)]


def test_balanced_offsets_power_law():
    P = nb.gen.powerlaw(20_000, max_deg=4000, seed=3)
    ip, tot = oracle.intprod(P, P)
    for world in (2, 3, 4, 8):
        off = nd.balanced_offsets(ip, world)
        assert off[0] == 0 and off[-1] == P.nrows and all(a <= b for a, b in zip(off, off[1:]))
        work = [int(ip[a:b].sum()) for a, b in zip(off, off[1:])]
        assert max(work) <= tot / world + ip.max()
        # the reference's split by row count is less even on this matrix
        even = nd.row_offsets(P.nrows, world)
        assert max(work) <= max(int(ip[a:b].sum()) for a, b in zip(even, even[1:]))
    assert nd.balanced_offsets([0, 0, 0], 2) == nd.row_offsets(3, 2)
    assert nd.balanced_offsets([], 4) == [0, 0, 0, 0, 0]


def test_row_offsets_match_reference_split():
    assert nd.row_offsets(10, 3) == [0, 3, 6, 10]
    assert nd.row_offsets(7, 1) == [0, 7]
    assert nd.row_offsets(5, 5) == [0, 1, 2, 3, 4, 5]
