"""Graph-file ingest on the device against the oracle's reader (itself pinned
to the reference's init_from_mtx by test_ingest_cpu.py): CSR arrays
bit-exact, at several piece sizes so lines straddle piece boundaries; the
error paths; the CSR cache; and the matrices in use (SpMV, BFS through
lablas::Matrix::init_from_mtx)."""
import numpy as np
import pytest

from gb_kun_b200 import graphgen as gg
from test_ingest_cpu import EDGE_FILE, csr_of, shuffled, write_case, CASES

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def capi():
    from gb_kun_b200 import capi
    capi.init(0)
    return capi


@pytest.fixture(scope="module")
def O():
    from oracle.cpu import Oracle
    return Oracle()


PIECES = [None, "4096", "257"]  # default 64 MiB, and pieces far smaller than the files


def read(capi, path, piece, monkeypatch, dtype="f32"):
    if piece:
        monkeypatch.setenv("GBK_INGEST_PIECE_BYTES", piece)
    else:
        monkeypatch.delenv("GBK_INGEST_PIECE_BYTES", raising=False)
    A = capi.Matrix.from_file(path, dtype=dtype)
    rp, col, val = A.download_csr()
    return A, rp, col, val


@pytest.mark.parametrize("piece", PIECES)
@pytest.mark.parametrize("case", CASES)
def test_mtx_matches_oracle(tmp_path, capi, O, monkeypatch, case, piece):
    f = tmp_path / "g.mtx"
    n, m, s, d = write_case(f, case)
    A, rp, col, val = read(capi, f, piece, monkeypatch)
    on, om, orp, ocol = O.read_graph_file(f)
    assert (A.n, A.ncols, A.nnz) == (on, om, len(ocol))
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.all(val == 1.0)


@pytest.mark.parametrize("piece", [None, "1024", "48"])
def test_mtxbin_matches_oracle(tmp_path, capi, O, monkeypatch, piece):
    g = gg.rmat(10, 8, seed=6)
    s, d = shuffled(g, 3)
    f = tmp_path / "g.mtxbin"
    gg.write_mtxbin(f, g.n, g.n, s, d)
    A, rp, col, val = read(capi, f, piece, monkeypatch, dtype="i32")
    _, _, orp, ocol = O.read_graph_file(f)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert val.dtype == np.int32 and np.all(val == 1)


@pytest.mark.parametrize("piece", [None, "64", "100"])
def test_edge_lines(tmp_path, capi, O, monkeypatch, piece):
    """CRLF, tabs, value column, '+', blank / comment lines between entries, lines past nnz (one of
    them malformed: not read, so not an error), and no newline after the last line."""
    f = tmp_path / "e.mtx"
    f.write_text(EDGE_FILE.rstrip("\n"))
    A, rp, col, _ = read(capi, f, piece, monkeypatch)
    _, _, orp, ocol = O.read_graph_file(f)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)


@pytest.mark.parametrize("body,line", [
    ("3 3 2\n1 2\n2 x\n", 2),
    ("3 3 2\n1 2\n2 4\n", 2),
    ("3 3 2\n0 1\n1 1\n", 1),
    ("3 3 2\n1 2x 3\n1 1\n", 1),
    ("3 3 2\n12345678901234567890 1\n1 1\n", 1),
])
def test_bad_lines_are_errors(tmp_path, capi, O, monkeypatch, body, line):
    f = tmp_path / "bad.mtx"
    f.write_text(body)
    with pytest.raises(ValueError):
        O.read_graph_file(f)
    for piece in (None, "64"):
        with pytest.raises(capi.GbkError) as e:
            read(capi, f, piece, monkeypatch)
        assert e.value.status == 5 and f"data line {line}" in str(e.value)


@pytest.mark.parametrize("body,what", [
    ("3 3 3\n1 2\n2 3\n", "unexpected end"),
    ("3 3\n1 2\n", "size line"),
    ("% only comments\n", "size line"),
])
def test_truncated_and_bad_headers(tmp_path, capi, monkeypatch, body, what):
    f = tmp_path / "bad.mtx"
    f.write_text(body)
    with pytest.raises(capi.GbkError) as e:
        read(capi, f, None, monkeypatch)
    assert e.value.status == 5 and what in str(e.value)


def test_other_errors(tmp_path, capi, monkeypatch):
    with pytest.raises(capi.GbkError) as e:
        capi.Matrix.from_file(tmp_path / "absent.mtx")
    assert e.value.status == 5
    (tmp_path / "g.txt").write_text("1 1 0\n")
    with pytest.raises(capi.GbkError) as e:
        capi.Matrix.from_file(tmp_path / "g.txt")
    assert e.value.status == 21
    long = tmp_path / "long.mtx"
    long.write_text("3 3 1\n" + " " * 200 + "1 1\n")
    with pytest.raises(capi.GbkError) as e:
        read(capi, long, "64", monkeypatch)
    assert "longer than" in str(e.value)
    short = tmp_path / "short.mtxbin"
    gg.write_mtxbin(short, 4, 4, np.array([0, 1], np.int32), np.array([1, 2], np.int32))
    short.write_bytes(short.read_bytes()[:-8])
    with pytest.raises(capi.GbkError) as e:
        capi.Matrix.from_file(short)
    assert "unexpected end" in str(e.value)
    bad = tmp_path / "bad.mtxbin"
    gg.write_mtxbin(bad, 4, 4, np.array([0, 7], np.int32), np.array([1, 2], np.int32))
    with pytest.raises(capi.GbkError) as e:
        capi.Matrix.from_file(bad)
    assert "entry 2" in str(e.value)


def test_empty_matrix(tmp_path, capi):
    f = tmp_path / "z.mtx"
    f.write_text("%%MatrixMarket matrix coordinate pattern general\n7 7 0\n")
    A = capi.Matrix.from_file(f)
    rp, col, _ = A.download_csr()
    assert A.nnz == 0 and np.array_equal(rp, np.zeros(8, np.int32))


def test_csr_cache_round_trip(tmp_path, capi):
    g = gg.rmat(12, 8, seed=9)
    val = gg.values_f32(g, seed=1)
    A = capi.Matrix.from_graph(g, val)
    f = tmp_path / "g.gbkcsr"
    A.save_csr(f)
    inf = capi.file_info(f)
    assert (inf.nrows, inf.ncols, inf.nnz, inf.kind, inf.vtype) == (g.n, g.n, g.nnz, 2, 0)
    for B in (capi.Matrix.load_csr(f), capi.Matrix.from_file(f)):
        rp, col, v = B.download_csr()
        assert np.array_equal(rp, g.row_ptr) and np.array_equal(col, g.col) and np.array_equal(v, val)


def test_corrupt_csr_cache_is_rejected(tmp_path, capi):
    g = gg.rmat(8, 4, seed=2)
    A = capi.Matrix.from_graph(g)
    f = tmp_path / "g.gbkcsr"
    A.save_csr(f)
    raw = bytearray(f.read_bytes())
    col0 = 64 + 4 * (g.n + 1)
    raw[col0:col0 + 4] = np.array([g.n + 5], np.int32).tobytes()  # a column past the end
    bad = tmp_path / "bad.gbkcsr"
    bad.write_bytes(bytes(raw))
    with pytest.raises(capi.GbkError) as e:
        capi.Matrix.load_csr(bad)
    assert "corrupt" in str(e.value)
    (tmp_path / "cut.gbkcsr").write_bytes(bytes(raw[:col0 + 8]))
    with pytest.raises(capi.GbkError):
        capi.Matrix.load_csr(tmp_path / "cut.gbkcsr")
    (tmp_path / "magic.gbkcsr").write_bytes(b"NOTACSR!" + bytes(raw[8:]))
    with pytest.raises(capi.GbkError):
        capi.Matrix.load_csr(tmp_path / "magic.gbkcsr")


@pytest.mark.parametrize("piece", [None, "1048576"])
def test_scale18_file_equals_generator(tmp_path, capi, monkeypatch, piece):
    """A file of about 50 MB in row order reads back as the generator's CSR."""
    g = gg.rmat(18, 16, seed=42)
    s, d = gg.edge_list(g)
    f = tmp_path / "g.mtx"
    gg.write_mtx(f, g.n, g.n, s, d)
    _, rp, col, _ = read(capi, f, piece, monkeypatch)
    assert np.array_equal(rp, g.row_ptr) and np.array_equal(col, g.col)


def test_spmv_on_matrix_from_file(tmp_path, capi, O):
    g = gg.rmat(13, 8, seed=11)
    s, d = shuffled(g, 4)
    f = tmp_path / "g.mtx"
    gg.write_mtx(f, g.n, g.n, s, d)
    A = capi.Matrix.from_file(f)
    x = gg.vector_f32(g.n, seed=2)
    dy = torch.zeros(g.n, device="cuda")
    A.mxv(torch.from_numpy(x).cuda(), dy)
    ref = O.spmv_f64(g, np.ones(g.nnz, np.float32), x)
    got = dy.cpu().numpy().astype(np.float64)
    assert np.abs(got - ref).sum() / np.abs(ref).sum() < 1e-6


def test_lablas_graph_from_file(tmp_path, O):
    from gb_kun_b200 import lablas_capi as L
    g = gg.rmat(12, 8, seed=12, undirected=True)
    s, d = shuffled(g, 5)
    f = tmp_path / "g.mtx"
    gg.write_mtx(f, g.n, g.n, s, d)
    G = L.Graph.from_file(f)
    src = int(gg.sources(g, 1, seed=3)[0])
    levels, _ = G.bfs(src)
    assert np.array_equal(levels, O.bfs(g, src))
    rect = tmp_path / "r.mtx"
    gg.write_mtx(rect, 5, 4, np.array([0], np.int32), np.array([1], np.int32))
    with pytest.raises(L.LablasError):
        L.Graph.from_file(rect)
