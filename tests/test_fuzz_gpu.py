"""Random small products through the GPU path against the oracle (hypothesis):
uneven row lengths (empty rows included), unsorted and duplicate B columns,
any shape; and the same pairs in one batched call and in a replayed plan."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import nsp_b200 as nb
import oracle
from nsp_b200.csr import HostCSR

from conftest import assert_close, assert_same_structure

pytestmark = pytest.mark.gpu


def random_csr(rng, n, m, dmax, unsorted=False, dup=False):
    deg = rng.integers(0, dmax + 1, n) if m else np.zeros(n, np.int64)
    deg = np.minimum(deg, m)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(deg)
    cols = []
    for d in deg:
        c = np.sort(rng.choice(m, int(d), replace=False)) if d else np.zeros(0, np.int64)
        if unsorted and d > 1:
            rng.shuffle(c)
        if dup and d > 1:
            c[-1] = c[0]
        cols.append(c)
    col = np.concatenate(cols).astype(np.int32) if n else np.zeros(0, np.int32)
    return HostCSR(n, m, rp, col, rng.uniform(-1, 1, int(rp[-1])))


shapes = st.tuples(st.integers(0, 300), st.integers(1, 400), st.integers(1, 500),
                   st.integers(0, 60), st.integers(0, 40), st.booleans(), st.booleans(),
                   st.integers(0, 2**31 - 1))


def check(got, A, B):
    rp, col, val = oracle.spgemm(A, B)
    h = got if isinstance(got, HostCSR) else got.to_host()
    assert (h.nrows, h.ncols) == (A.nrows, B.ncols)
    assert_same_structure(h.rowptr, h.col, rp, col)
    assert_close(h.val, val, oracle.absbound(A, B, rp, col))


@settings(max_examples=60, deadline=None, suppress_health_check=list(HealthCheck))
@given(shapes)
def test_random_products(cuda, s):
    n, k, m, da, db, unsorted, dup, seed = s
    rng = np.random.default_rng(seed)
    A = random_csr(rng, n, k, da)
    B = random_csr(rng, k, m, db, unsorted, dup)
    check(nb.spgemm(A.to_device(), B.to_device()), A, B)
    rp, col, val = nb.spgemm_host(A, B, nblocks=1 + seed % 5)  # host operands and result
    check(HostCSR(A.nrows, B.ncols, rp, col, val), A, B)


@settings(max_examples=10, deadline=None, suppress_health_check=list(HealthCheck))
@given(st.lists(shapes, min_size=1, max_size=12))
def test_random_batches(cuda, ss):
    pairs = []
    for n, k, m, da, db, unsorted, dup, seed in ss:
        rng = np.random.default_rng(seed)
        pairs.append((random_csr(rng, n, k, da), random_csr(rng, k, m, db, unsorted, dup)))
    dA = [a.to_device() for a, _ in pairs]
    dB = [b.to_device() for _, b in pairs]
    Cs = nb.spgemm_batched(dA, dB)
    for got, (A, B) in zip(Cs, pairs):
        check(got, A, B)
    plan = nb.Plan(dA, dB, max_group=1 + len(pairs) // 3)  # several groups in one graph
    plan.execute()
    for got, (A, B) in zip(plan.C, pairs):
        check(got, A, B)
