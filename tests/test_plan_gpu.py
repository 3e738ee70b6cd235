"""Plans (nspb_plan_*): symbolic once, numeric replayed from a CUDA graph with
the inputs' current values; results against the oracle after every change
of values, for one product and for a batch."""
import numpy as np
import pytest
import torch

import nsp_b200 as nb
import oracle
from nsp_b200 import amg
from nsp_b200.csr import HostCSR

from conftest import assert_bitwise, assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def host_of(d):
    return HostCSR(d.nrows, d.ncols, d.rowptr.cpu().numpy(), d.col.cpu().numpy(),
                   d.val.double().cpu().numpy())


def check(got, A, B, exact=True):
    rp, col, val = oracle.spgemm(A, B)
    h = host_of(got)
    assert_same_structure(h.rowptr, h.col, rp, col)
    if exact:
        assert_bitwise(h.val, val)
    else:
        assert_close(h.val, val, oracle.absbound(A, B, rp, col))


def test_single_product_replay(cuda):
    A = nb.gen.random(4000, 3000, 1, 40, seed=1)
    B = nb.gen.random(3000, 2500, 1, 12, seed=2)
    dA, dB = A.to_device(), B.to_device()
    plan = nb.Plan([dA], [dB])
    assert plan.stats["nnz"] == plan.C[0].nnz > 0
    check(plan.C[0], A, B)
    for k in range(3):  # new values in place, same structure
        dA.val.mul_(-1.5).add_(0.25)
        dB.val.mul_(0.5)
        plan.execute()
        check(plan.C[0], host_of(dA), host_of(dB))


def test_batch_replay_amg_and_random(cuda):
    pairs = amg.amg_batch(L=15, levels=3) + amg.random_batch(20, 200, 3000, 1, 16, seed=4)
    dA = [a.to_device() for a, _ in pairs]
    dB = [b.to_device() for _, b in pairs]
    plan = nb.Plan(dA, dB)
    for got, (A, B) in zip(plan.C, pairs):
        check(got, A, B, exact=False)
    for d in dA:
        d.val.mul_(2.0).sub_(1.0)
    plan.execute()
    for got, a, b in zip(plan.C, dA, dB):
        check(got, host_of(a), host_of(b), exact=False)
    first = [c.val.clone() for c in plan.C]
    plan.execute()
    # rows of at most 512 entries accumulate in a fixed order: replays agree bit for bit
    if sum(plan.stats["num_bins"][6:]) == 0:
        for c, f in zip(plan.C, first):
            assert torch.equal(c.val, f)


def test_fp32c_plan(cuda):
    A = nb.gen.stencil(10, npts=27, fp32=True)
    d32 = HostCSR(A.nrows, A.ncols, A.rowptr, A.col, A.val.astype(np.float32)).to_device()
    plan = nb.Plan([d32], [d32], precision="fp32c")
    rp, col, val = oracle.spgemm(A, A)
    got = host_of(plan.C[0])
    assert_same_structure(got.rowptr, got.col, rp, col)
    bound = oracle.absbound(A, A, rp, col)
    assert np.all(np.abs(got.val - val) <= 1e-10 * bound + 1e-300)
    d32.val.mul_(0.5)
    plan.execute()
    got = host_of(plan.C[0])
    assert np.all(np.abs(got.val - 0.25 * val) <= 1e-10 * 0.25 * bound + 1e-300)


def test_views_keep_plan_alive(cuda):
    A = nb.gen.random(500, 400, 1, 9, seed=7)
    dA = A.to_device()
    plan = nb.Plan([dA], [nb.gen.random(400, 300, 1, 5, seed=8).to_device()])
    col = plan.C[0].col
    del plan  # the view still references the plan's arrays
    assert col.numel() > 0 and int(col.max()) < 300


def test_plan_several_groups_one_graph(cuda):
    # at most 3 products per block-diagonal group: 4 groups (one of a single
    # product) captured in one graph
    pairs = amg.random_batch(10, 300, 4000, 1, 14, seed=11)
    dA = [a.to_device() for a, _ in pairs]
    dB = [b.to_device() for _, b in pairs]
    plan = nb.Plan(dA, dB, max_group=3)
    for got, (A, B) in zip(plan.C, pairs):
        check(got, A, B, exact=False)
    for d in dB:
        d.val.mul_(-3.0)
    plan.execute()
    for got, a, b in zip(plan.C, dA, dB):
        check(got, host_of(a), host_of(b), exact=False)
    Cs = nb.spgemm_batched(dA, dB, max_group=2)
    for got, a, b in zip(Cs, dA, dB):
        check(got, host_of(a), host_of(b), exact=False)
