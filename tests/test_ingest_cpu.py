"""Graph-file ingest, CPU side: the C oracle's reader against the reference's
own Matrix<T>::init_from_mtx (src/backend/matrix/read_file.hpp:565-617) on
generated files, the oracle on the lines the reference cannot read, and the
oracle's error codes."""
import numpy as np
import pytest

from gb_kun_b200 import graphgen as gg
from oracle.cpu import Oracle, Reference

needs_ref = pytest.mark.skipif(not Reference.available(), reason="reference CPU build absent")


@pytest.fixture(scope="module")
def O():
    return Oracle()


@pytest.fixture(scope="module")
def R():
    return Reference()


def shuffled(g, seed):
    s, d = gg.edge_list(g)
    p = np.random.default_rng(seed).permutation(len(s))
    return s[p], d[p]


def csr_of(nrows, s, d):
    """CSR with every row in the given (file) order."""
    order = np.argsort(s, kind="stable")
    rp = np.zeros(nrows + 1, np.int64)
    np.add.at(rp, s.astype(np.int64) + 1, 1)
    return np.cumsum(rp).astype(np.int32), d[order].astype(np.int32)


def write_case(path, case):
    """(nrows, ncols, src, dst) of a named case, written to path."""
    rng = np.random.default_rng(7)
    if case == "rmat_shuffled_real":
        g = gg.rmat(11, 8, seed=3)
        s, d = shuffled(g, 1)
        gg.write_mtx(path, g.n, g.n, s, d, vals=rng.random(len(s)))
        return g.n, g.n, s, d
    if case == "er_pattern":
        g = gg.uniform(10, 6, seed=4)
        s, d = shuffled(g, 2)
        gg.write_mtx(path, g.n, g.n, s, d)
        return g.n, g.n, s, d
    if case == "duplicates":
        s = rng.integers(0, 50, 3000).astype(np.int32)
        d = rng.integers(0, 50, 3000).astype(np.int32)
        gg.write_mtx(path, 50, 50, s, d)
        return 50, 50, s, d
    if case == "rect":
        s = rng.integers(0, 300, 2000).astype(np.int32)
        d = rng.integers(0, 90, 2000).astype(np.int32)
        gg.write_mtx(path, 300, 90, s, d)
        return 300, 90, s, d
    if case == "empty_rows":
        s = (rng.integers(0, 40, 500) * 7).astype(np.int32)
        d = rng.integers(0, 280, 500).astype(np.int32)
        gg.write_mtx(path, 300, 300, s, d)
        return 300, 300, s, d
    raise ValueError(case)


CASES = ["rmat_shuffled_real", "er_pattern", "duplicates", "rect", "empty_rows"]


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_mtx(tmp_path, O, R, case):
    f = tmp_path / "g.mtx"
    n, m, s, d = write_case(f, case)
    on, oc, rp, col = O.read_graph_file(f)
    rn, rrp, rcol, rval, _ = R.graph_read(f)
    assert (on, oc) == (n, m) and rn == n
    assert np.array_equal(rp, rrp) and np.array_equal(col, rcol)  # same arrays, rows in file order
    assert np.all(rval == 1.0)                                    # EDGE_VAL
    erp, ecol = csr_of(n, s, d)
    assert np.array_equal(rp, erp) and np.array_equal(col, ecol)


@needs_ref
@pytest.mark.parametrize("case", ["rmat_shuffled_real", "duplicates"])
def test_oracle_matches_reference_mtxbin(tmp_path, O, R, case):
    """The reference orders a .mtxbin row by hash-map iteration (read_file.hpp:428-476), so rows are
    compared as multisets; the oracle keeps the file order."""
    n, m, s, d = write_case(tmp_path / "g.mtx", case)
    f = tmp_path / "g.mtxbin"
    gg.write_mtxbin(f, n, m, s, d)
    _, _, rp, col = O.read_graph_file(f)
    rn, rrp, rcol, _, _ = R.graph_read(f)
    assert rn == n and np.array_equal(rp, rrp)
    for i in range(n):
        assert np.array_equal(np.sort(col[rp[i]:rp[i + 1]]), np.sort(rcol[rrp[i]:rrp[i + 1]]))
    erp, ecol = csr_of(n, s, d)
    assert np.array_equal(rp, erp) and np.array_equal(col, ecol)


EDGE_FILE = (
    "%%MatrixMarket matrix coordinate real general\r\n"
    "% a comment\r\n"
    "%another\r\n"
    "5 4 6\r\n"
    "3 1 0.5\r\n"
    "\r\n"
    "  1\t4   2.0\r\n"
    "% a comment between entries\n"
    "+2 2\n"
    "5 3 1e-3\n"
    "3 2\n"
    "1 1\n"
    "4 4 this line is past nnz\n"
    "not an entry either\n"
)


def test_oracle_edge_lines(tmp_path, O):
    """CRLF, tabs, a value column, '+' signs, blank and comment lines between entries, lines past nnz."""
    f = tmp_path / "e.mtx"
    f.write_text(EDGE_FILE)
    n, m, rp, col = O.read_graph_file(f)
    s = np.array([3, 1, 2, 5, 3, 1]) - 1
    d = np.array([1, 4, 2, 3, 2, 1]) - 1
    erp, ecol = csr_of(5, s, d)
    assert (n, m) == (5, 4)
    assert np.array_equal(rp, erp) and np.array_equal(col, ecol)


@pytest.mark.parametrize("body,code,line", [
    ("3 3 2\n1 2\n2 x\n", 3, 2),          # malformed
    ("3 3 2\n1 2\n2 4\n", 3, 2),          # column outside 1..3
    ("3 3 2\n0 1\n1 1\n", 3, 1),          # ids are 1-based
    ("3 3 3\n1 2\n2 3\n", 4, 0),          # fewer entries than nnz
    ("3 3\n1 2\n", 2, 0),                 # size line without nnz
    ("% only comments\n", 2, 0),         # no size line
])
def test_oracle_errors(tmp_path, O, body, code, line):
    f = tmp_path / "bad.mtx"
    f.write_text(body)
    with pytest.raises(ValueError) as e:
        O.read_graph_file(f)
    assert e.value.args[0] == code
    if line:
        assert e.value.args[1] == line


def test_oracle_missing_file(tmp_path, O):
    with pytest.raises(ValueError) as e:
        O.read_graph_file(tmp_path / "absent.mtx")
    assert e.value.args[0] == 1


def test_writer_round_trip(tmp_path, O):
    g = gg.rmat(9, 8, seed=5)
    s, d = gg.edge_list(g)
    gg.write_mtx(tmp_path / "a.mtx", g.n, g.n, s, d)
    gg.write_mtxbin(tmp_path / "a.mtxbin", g.n, g.n, s, d)
    for f in ("a.mtx", "a.mtxbin"):
        _, _, rp, col = O.read_graph_file(tmp_path / f)
        assert np.array_equal(rp, g.row_ptr) and np.array_equal(col, g.col)
