"""Matrix files in the reference's formats (host code of libnspb.so).

The byte layouts are restated here with numpy structured dtypes, independently
of the C code: the binary COO header of int64 {nr, nc, nt} or {nr, nt} and
records {ii, jj, aa} with 1-based int64 or int32 indices
(src/READ_MATRIX_MPI.cpp:146-356), the writer's header {nr, nc} in the index
width followed by an int64 nt (main.cu:468-512), and the MatrixMarket text of
src/matrixIO.cu:299-339.
"""
import numpy as np
import pytest

import nsp_b200 as nb
from nsp_b200 import matio
from nsp_b200._lib import ERR_INVALID, ERR_IO
from nsp_b200.csr import HostCSR

REC8 = np.dtype([("ii", "<i8"), ("jj", "<i8"), ("aa", "<f8")])
REC4 = np.dtype([("ii", "<i4"), ("jj", "<i4"), ("aa", "<f8")])


def _records(M, dt):
    rows = np.repeat(np.arange(M.nrows), np.diff(M.rowptr))
    r = np.zeros(M.nnz, dt)
    r["ii"], r["jj"], r["aa"] = rows + 1, M.col + 1, M.val
    return r


def _same(a, b):
    assert a.nrows == b.nrows and a.ncols == b.ncols
    assert np.array_equal(a.rowptr, b.rowptr)
    assert np.array_equal(a.col, b.col)
    assert np.array_equal(a.val, b.val)


@pytest.fixture
def M():
    return nb.gen.random(300, 250, 1, 9, seed=5)  # no empty rows


@pytest.mark.parametrize("width", [8, 4])
def test_writer_layout(tmp_path, M, width):
    p = tmp_path / "m.bin"
    matio.write_coo_bin(p, M, index_bytes=width)
    raw = p.read_bytes()
    hdr_dt = np.dtype([("nr", f"<i{width}"), ("nc", f"<i{width}"), ("nt", "<i8")])
    hdr = np.frombuffer(raw[:hdr_dt.itemsize], hdr_dt)[0]
    assert (hdr["nr"], hdr["nc"], hdr["nt"]) == (M.nrows, M.ncols, M.nnz)
    rec = np.frombuffer(raw[hdr_dt.itemsize:], REC8 if width == 8 else REC4)
    assert np.array_equal(rec, _records(M, rec.dtype))


def test_binary_round_trip(tmp_path, M):
    p = tmp_path / "m.bin"
    matio.write_coo_bin(p, M)
    got, info = matio.read_coo_bin(p, info=True)
    _same(got, M)
    assert info["full_nrows"] == M.nrows and info["first_row"] == 0


def test_reader_header_type0_int32_records(tmp_path, M):
    p = tmp_path / "m.bin"
    with open(p, "wb") as f:
        f.write(np.array([M.nrows, M.nnz], "<i8").tobytes())
        f.write(_records(M, REC4).tobytes())
    got = matio.read_coo_bin(p, header_type=0, index_bytes=4)
    sq = HostCSR(M.nrows, M.nrows, M.rowptr, M.col, M.val)  # header_type 0: nc = nr
    _same(got, sq)


def test_reader_sorts_rows_stably_and_keeps_duplicates(tmp_path):
    rec = np.zeros(6, REC8)
    rec["ii"] = [1, 1, 1, 1, 2, 2]
    rec["jj"] = [5, 2, 5, 1, 3, 3]
    rec["aa"] = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
    p = tmp_path / "u.bin"
    with open(p, "wb") as f:
        f.write(np.array([2, 6, 6], "<i8").tobytes())
        f.write(rec.tobytes())
    got = matio.read_coo_bin(p)
    assert list(got.rowptr) == [0, 4, 6]
    assert list(got.col) == [0, 1, 4, 4, 2, 2]
    assert list(got.val) == [4.0, 2.0, 1.0, 3.0, 5.0, 6.0]


def test_rows_counted_from_first_stored_row(tmp_path):
    rec = np.zeros(3, REC8)
    rec["ii"], rec["jj"], rec["aa"] = [3, 3, 6], [1, 2, 2], [1.0, 2.0, 3.0]
    p = tmp_path / "f.bin"
    with open(p, "wb") as f:
        f.write(np.array([8, 4, 3], "<i8").tobytes())
        f.write(rec.tobytes())
    got, info = matio.read_coo_bin(p, info=True)
    assert got.nrows == 4 and info["first_row"] == 2 and info["full_nrows"] == 8
    assert list(got.rowptr) == [0, 2, 2, 2, 3]


def test_reader_errors(tmp_path):
    with pytest.raises(nb.NspbError) as e:
        matio.read_coo_bin(tmp_path / "missing.bin")
    assert e.value.status == ERR_IO
    p = tmp_path / "t.bin"
    with open(p, "wb") as f:  # header promises 5 records, file holds 2
        f.write(np.array([3, 3, 5], "<i8").tobytes())
        f.write(np.zeros(2, REC8).tobytes())
    with pytest.raises(nb.NspbError) as e:
        matio.read_coo_bin(p)
    assert e.value.status == ERR_IO
    for ii, jj in (([2, 1], [1, 1]), ([1, 1], [0, 1]), ([1, 1], [1, 4])):
        rec = np.zeros(2, REC8)
        rec["ii"], rec["jj"] = ii, jj
        with open(p, "wb") as f:  # rows out of order, column 0, column > nc
            f.write(np.array([3, 3, 2], "<i8").tobytes())
            f.write(rec.tobytes())
        with pytest.raises(nb.NspbError) as e:
            matio.read_coo_bin(p)
        assert e.value.status == ERR_INVALID


def test_empty_file_round_trip(tmp_path):
    E = HostCSR(4, 3, np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0))
    p = tmp_path / "e.bin"
    matio.write_coo_bin(p, E)
    got, info = matio.read_coo_bin(p, info=True)
    assert got.nrows == 0 and got.nnz == 0 and info["full_nrows"] == 4


def test_mtx_writer_text(tmp_path, M):
    p = tmp_path / "m.mtx"
    matio.write_mtx(p, M)
    lines = ["%%MatrixMarket matrix coordinate real general",
             "%d  %d %d " % (M.nrows, M.ncols, M.nnz)]
    for r in range(M.nrows):
        for t in range(M.rowptr[r], M.rowptr[r + 1]):
            lines.append("%d   %d  %g" % (r + 1, M.col[t] + 1, M.val[t]))
    assert p.read_text() == "\n".join(lines) + "\n"


def test_ascii_reader_reads_writer_output(tmp_path, M):
    p = tmp_path / "m.mtx"
    matio.write_mtx(p, M)
    got = matio.read_coo_ascii(p)
    rounded = np.array([float("%g" % v) for v in M.val])
    _same(got, HostCSR(M.nrows, M.ncols, M.rowptr, M.col, rounded))


def test_ascii_two_number_header(tmp_path):
    p = tmp_path / "s.txt"
    p.write_text("% comment\n3 2\n1 1 2.5\n3 3 -1\n")
    got = matio.read_coo_ascii(p)
    assert got.nrows == 3 and got.ncols == 3
    assert list(got.rowptr) == [0, 1, 1, 2] and list(got.col) == [0, 2]
    assert list(got.val) == [2.5, -1.0]
