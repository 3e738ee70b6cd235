"""The row-template criterion on the CPU (numpy), independent of the kernels:
B row shift bits (bit k: B row k is row k-1 with every column moved by one
amount) and the per-row test the entry-map kernels apply before reusing a
row's count, map and sort. Whenever the test accepts a pair of rows, their
intermediate-product column sequences must differ by one constant, so their
first-appearance maps are equal and their sorted column orders correspond;
and on a stencil the test must accept most neighbouring rows (it is not
vacuous). The GPU tests check the kernels themselves against the oracle."""
import numpy as np
import pytest

import nsp_b200.gen as gen
from test_row_template_gpu import perturb


def shift_bits(B):
    rp, col = B.rowptr, B.col
    bits = np.zeros(B.nrows, bool)
    for k in range(1, B.nrows):
        a0, a1, b0, b1 = rp[k - 1], rp[k], rp[k], rp[k + 1]
        if a1 - a0 != b1 - b0:
            continue
        bits[k] = b1 == b0 or np.all(col[b0:b1] - col[b0] == col[a0:a1] - col[a0])
    return bits


def same_run(bits, k, kt):
    """B rows k and kt in one run of shifted rows (followed over 31 rows at most)."""
    if k == kt:
        return True
    lo, hi = min(k, kt) + 1, max(k, kt)
    return hi - lo < 31 and bool(np.all(bits[lo:hi + 1]))


def b_rows(A, B, i):
    ks = A.col[A.rowptr[i]:A.rowptr[i + 1]]
    return [(int(k), int(B.rowptr[k]), int(B.rowptr[k + 1])) for k in ks]


def first_col(B, s, e):
    return int(B.col[s]) if e > s else None


def accept(A, B, bits, i, t):
    """The kernels' test: same A length, each B row of the template's length,
    and every non-empty B row in one run with the template's, moved by the
    shift of the first non-empty pair."""
    ri, rt = b_rows(A, B, i), b_rows(A, B, t)
    if len(ri) != len(rt):
        return False
    shift = None
    for (k, s, e), (kt, st, et) in zip(ri, rt):
        if e - s != et - st:
            return False
        if e == s:
            continue
        d = int(B.col[s]) - int(B.col[st])
        if shift is None:
            shift = d
        if d != shift or not same_run(bits, k, kt):
            return False
    return True


def products(A, B, i):
    return np.concatenate([B.col[s:e] for _, s, e in b_rows(A, B, i)] or [np.zeros(0, np.int32)])


def first_appearance(seq):
    seen = {}
    return [seen.setdefault(int(c), len(seen)) for c in seq]


def check_pairs(A, B, pairs):
    bits = shift_bits(B)
    accepted = 0
    for i, t in pairs:
        if not accept(A, B, bits, i, t):
            continue
        accepted += 1
        pi, pt = products(A, B, i).astype(np.int64), products(A, B, t).astype(np.int64)
        assert len(pi) == len(pt)
        if len(pi):
            assert np.all(pi - pt == pi[0] - pt[0]), (i, t)
            assert first_appearance(pi) == first_appearance(pt)
            assert np.array_equal(np.argsort(pi, kind="stable"), np.argsort(pt, kind="stable"))
    return accepted


def neighbour_pairs(n, dists=(1, 2, 5, 16), stride=7):
    return [(i, i - d) for i in range(0, n, stride) for d in dists if i - d >= 0]


@pytest.mark.parametrize("npts", [7, 27])
def test_stencil_neighbours_accepted_and_sound(npts):
    A = gen.stencil(14, npts=npts)
    check_pairs(A, A, neighbour_pairs(A.nrows))  # sound at every distance
    # adjacent rows of a line share their pattern away from the grid's faces:
    # for 14 points a line, 9 of 14 rows follow a row of the same pattern
    # (the 27-point pattern reaches two rows into each face)
    nxt = neighbour_pairs(A.nrows, dists=(1,), stride=1)
    assert check_pairs(A, A, nxt) > 0.5 * len(nxt)


@pytest.mark.parametrize("frac,seed", [(0.02, 1), (0.2, 2)])
def test_moved_columns_never_accepted_wrongly(frac, seed):
    A = gen.stencil(12, npts=27)
    P = perturb(A, frac, seed)
    for X, Y in ((P, A), (A, P), (P, P)):
        check_pairs(X, Y, neighbour_pairs(X.nrows, stride=5))


def test_random_rows_sound():
    A = gen.random(600, 500, 0, 12, seed=3)
    B = gen.random(500, 400, 0, 6, seed=4)
    check_pairs(A, B, [(i, t) for i in range(0, 600, 3) for t in range(max(0, i - 8), i)])


def test_shift_bits_are_needed():
    # a weakened test that ignores the shift bits (lengths and first columns
    # only) accepts rows whose columns differ: the bits carry the soundness
    A = gen.stencil(12, npts=27)
    P = perturb(A, 0.2, seed=2)
    every = np.ones(P.nrows, bool)
    unsound = 0
    for i, t in neighbour_pairs(A.nrows, dists=(1, 2), stride=1):
        if not accept(A, P, every, i, t):
            continue
        pi, pt = products(A, P, i).astype(np.int64), products(A, P, t).astype(np.int64)
        unsound += bool(len(pi)) and not np.all(pi - pt == pi[0] - pt[0])
    assert unsound > 0
