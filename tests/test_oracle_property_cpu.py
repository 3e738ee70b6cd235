"""Property test of the oracle against an independent pure-Python Gustavson
product: random small CSR operands with empty rows, unsorted rows, duplicate
columns (summed) and cancellations (kept as explicit zeros). Both add the
rounded products a_ik * b_kj in A-row order, so values agree bit for bit."""
import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

import oracle
from nsp_b200.csr import HostCSR


@st.composite
def csr(draw, nrows, ncols):
    rows = []
    for _ in range(nrows):
        k = draw(st.integers(0, min(ncols, 6)) if ncols else st.just(0))
        cols = draw(st.lists(st.integers(0, max(ncols - 1, 0)), min_size=k, max_size=k))
        vals = draw(st.lists(st.sampled_from([-2.0, -1.0, -0.5, 0.25, 1.0, 3.0, 0.1, -0.3]),
                             min_size=k, max_size=k))
        rows.append(list(zip(cols, vals)))
    rp = np.zeros(nrows + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.array([c for r in rows for c, _ in r], np.int32)
    val = np.array([v for r in rows for _, v in r], np.float64)
    return HostCSR(nrows, ncols, rp, col, val)


@st.composite
def pair(draw):
    n = draw(st.integers(0, 12))
    k = draw(st.integers(0, 10))
    m = draw(st.integers(0, 12))
    return draw(csr(n, k)), draw(csr(k, m))


def gustavson(A, B):
    rp, col, val = [0], [], []
    for i in range(A.nrows):
        acc = {}
        for t in range(A.rowptr[i], A.rowptr[i + 1]):
            k, a = int(A.col[t]), float(A.val[t])
            for u in range(B.rowptr[k], B.rowptr[k + 1]):
                j = int(B.col[u])
                acc[j] = acc.get(j, 0.0) + a * float(B.val[u])
        for j in sorted(acc):
            col.append(j)
            val.append(acc[j])
        rp.append(len(col))
    return np.array(rp), np.array(col, np.int64), np.array(val)


@settings(max_examples=150, deadline=None)
@given(pair())
def test_oracle_equals_plain_gustavson(ab):
    A, B = ab
    rp, col, val = oracle.spgemm(A, B)
    wrp, wcol, wval = gustavson(A, B)
    assert np.array_equal(np.asarray(rp, np.int64), wrp)
    assert np.array_equal(np.asarray(col, np.int64), wcol)
    assert np.array_equal(np.asarray(val).view(np.int64), wval.view(np.int64))
