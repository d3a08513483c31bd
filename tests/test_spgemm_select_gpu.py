"""Unmasked SpGEMM (gbk_mxm) and select on the device against the reference's
own SpMSpM_unmasked_ikj and select (harness, pinned to dense numpy by
test_spgemm_select_cpu.py) and dense numpy.  The reference orders a row of
an unmasked product by hash-map iteration, so rows are compared sorted."""
import numpy as np
import pytest

from gb_kun_b200 import graphgen as gg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def capi():
    from gb_kun_b200 import capi
    capi.init(0)
    return capi


@pytest.fixture(scope="module")
def R():
    from oracle.cpu import Reference
    if not Reference.available():
        pytest.skip("reference CPU build absent")
    return Reference()


def sorted_rows(rp, col, val):
    n = len(rp) - 1
    order = np.lexsort((col, np.repeat(np.arange(n), np.diff(rp))))
    return col[order], val[order]


def dense(nr, nc, rp, col, val):
    A = np.zeros((nr, nc))
    A[np.repeat(np.arange(nr), np.diff(rp)), col] = val
    return A


GRAPHS = {"rmat10": lambda: gg.rmat(10, 8, seed=3), "er9": lambda: gg.uniform(9, 6, seed=4),
          "rmat9u": lambda: gg.rmat(9, 8, seed=5, undirected=True)}
SEMIRINGS = {"plus_times": 0, "lor_land": 1, "min_plus": 6, "plus_one": 10}


@pytest.mark.parametrize("block", [None, "1", "997"])
@pytest.mark.parametrize("sr", sorted(SEMIRINGS))
@pytest.mark.parametrize("gname", sorted(GRAPHS))
def test_mxm_matches_reference(capi, R, monkeypatch, gname, sr, block):
    if block:
        monkeypatch.setenv("GBK_MXM_BLOCK_PRODUCTS", block)
    else:
        monkeypatch.delenv("GBK_MXM_BLOCK_PRODUCTS", raising=False)
    g = GRAPHS[gname]()
    val = gg.values_f32(g, seed=7) + np.float32(0.25)  # no zero values
    if sr == "lor_land":
        val = np.ones(g.nnz, np.float32)
    A = capi.Matrix.from_graph(g, val)
    C = A.mxm(A, semiring=sr)
    rp, col, v = C.download_csr()
    rrp, rcol, rv, _ = R.mxm(g, val, SEMIRINGS[sr])
    assert np.array_equal(rp, rrp)
    c1, v1 = sorted_rows(rp, col, v)
    c2, v2 = sorted_rows(rrp, rcol, rv)
    assert np.array_equal(c1, c2)
    assert np.allclose(v1, v2, rtol=2e-6, atol=0)
    # ours: every row already column-sorted
    rows = np.repeat(np.arange(g.n), np.diff(rp))
    assert np.all(np.diff(rows * (g.n + 1) + col) > 0)


def test_mxm_int_and_rectangular(capi):
    rng = np.random.default_rng(1)
    a = gg.from_edges(300, rng.integers(0, 300, 4000), rng.integers(0, 300, 4000))
    av = rng.integers(-3, 4, a.nnz).astype(np.int32)
    # B: 300 x 170 (rows of a's columns, fewer columns)
    bs, bd = rng.integers(0, 300, 3000), rng.integers(0, 170, 3000)
    order = np.lexsort((bd, bs))
    pairs = np.unique(np.stack([bs[order], bd[order]], 1), axis=0)
    brp = np.zeros(301, np.int32)
    np.add.at(brp, pairs[:, 0] + 1, 1)
    brp = np.cumsum(brp).astype(np.int32)
    bcol = pairs[:, 1].astype(np.int32)
    bv = rng.integers(-3, 4, len(bcol)).astype(np.int32)
    A = capi.Matrix(a.row_ptr, a.col, av)
    B = capi.Matrix(brp, bcol, bv, ncols=170)
    C = A.mxm(B)
    rp, col, v = C.download_csr()
    D = dense(300, 300, a.row_ptr, a.col, av) @ dense(300, 170, brp, bcol, bv)
    assert (C.n, C.ncols) == (300, 170)
    rows = np.repeat(np.arange(300), np.diff(rp))
    assert np.array_equal(D[rows, col], v) and rp[-1] == np.count_nonzero(D)  # zeros dropped
    M = A.mxm(B, semiring="min_plus")
    rp, col, v = M.download_csr()
    rows = np.repeat(np.arange(300), np.diff(rp))
    Ad, Bd = dense(300, 300, a.row_ptr, a.col, av), dense(300, 170, brp, bcol, bv)
    Pa, Pb = dense(300, 300, a.row_ptr, a.col, 1), dense(300, 170, brp, bcol, 1)
    big = 1e18
    S = np.min(np.where((Pa[:, :, None] > 0) & (Pb[None, :, :] > 0), Ad[:, :, None] + Bd[None, :, :], big), axis=1)
    assert np.array_equal(S[rows, col], v)
    assert np.count_nonzero((S < big) & (S != 0)) == rp[-1]


def test_mxm_errors(capi):
    g = gg.rmat(6, 4, seed=1)
    A = capi.Matrix.from_graph(g)
    Ai = capi.Matrix.from_graph(g, np.ones(g.nnz, np.int32))
    with pytest.raises(capi.GbkError) as e:
        A.mxm(Ai)
    assert e.value.status == 7  # domain mismatch
    B = capi.Matrix(np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32), ncols=5)
    with pytest.raises(capi.GbkError) as e:
        A.mxm(B)
    assert e.value.status == 8
    with pytest.raises(capi.GbkError) as e:
        A.mxm(A, semiring="custom_less_plus")
    assert e.value.status == 21


@pytest.mark.parametrize("op,code,thunk", [("tril", 0, -1), ("triu", 1, 1), ("diag", 2, 0), ("offdiag", 3, 0),
                                           ("tril", 0, 3), ("value_gt", 6, 0.5), ("value_le", 9, 0.25)])
def test_select_matrix_matches_reference(capi, R, op, code, thunk):
    g = gg.rmat(10, 8, seed=9)
    val = gg.values_f32(g, seed=2)
    A = capi.Matrix.from_graph(g, val)
    rp, col, v = A.select(op, thunk).download_csr()
    rrp, rcol, rv = R.select_matrix(g, val, code, thunk)
    assert np.array_equal(rp, rrp) and np.array_equal(col, rcol) and np.array_equal(v, rv)


@pytest.mark.parametrize("op,thunk", [("tril", -5), ("value_ge", 0.5), ("value_ne", 0.0)])
@pytest.mark.parametrize("masking", ["none", "mask", "comp", "replace"])
def test_select_vector(capi, op, thunk, masking):
    n = 1000
    rng = np.random.default_rng(3)
    u = rng.random(n).astype(np.float32)
    u[::7] = 0
    w0 = rng.random(n).astype(np.float32)
    mask = (rng.random(n) < 0.4).astype(np.float32)
    i = np.arange(n)
    keep = {"tril": 0 <= i + thunk, "value_ge": u >= thunk, "value_ne": u != thunk}[op]
    r = np.where(keep, u, 0).astype(np.float32)
    w = torch.from_numpy(w0.copy()).cuda()
    if masking == "none":
        capi.select_vector(w, torch.from_numpy(u).cuda(), op, thunk, accum="plus")
        expect = w0 + r
    else:
        sel = mask != 0
        if masking == "comp":
            sel = ~sel
        capi.select_vector(w, torch.from_numpy(u).cuda(), op, thunk, accum="plus", mask=torch.from_numpy(mask).cuda(),
                           mask_mode="comp" if masking == "comp" else "default", replace=(masking == "replace"))
        expect = np.where(sel, w0 + r, 0 if masking == "replace" else w0)
    assert np.allclose(w.cpu().numpy(), expect, rtol=1e-6)


@pytest.mark.parametrize("method", range(7))
def test_triangle_count_methods_match_reference(R, method):
    """Every LAGr_TriangleCount method through lablas:: (select + masked SpGEMM) against the reference's
    own method; the reference's L / U keep A's structure, so all methods give the Burkhardt count."""
    from gb_kun_b200 import lablas_capi as L
    g = gg.rmat(11, 8, seed=4, undirected=True)
    G = L.Graph(g)
    got, _ = G.tc_method(method)
    ref, _ = R.tc_method(g, method)
    assert got == ref
    assert got == G.tc()[0]


def test_coo_format_spmv(capi):
    """COO (set_preferred_matrix_format(COO)) is stored as CSR: same SpMV as CSR."""
    from gb_kun_b200 import lablas_capi as L
    g = gg.rmat(11, 8, seed=6)
    val = gg.values_f32(g, seed=1)
    x = gg.vector_f32(g.n, seed=2)
    G = L.Graph(g)
    y_coo, _ = G.spmv(val, x, fmt=1)
    y_csr, _ = G.spmv(val, x, fmt=0)
    assert np.array_equal(y_coo, y_csr)


def test_triangle_count_entry(capi, R):
    """gbk_triangle_count: the oriented count on a simple undirected graph and the masked-product formula
    on a directed one and one with self loops, each against the reference's Burkhardt count."""
    und = gg.rmat(12, 8, seed=7, undirected=True)
    A = capi.Matrix.from_graph(und, np.ones(und.nnz, np.int32))
    assert A.triangle_count() == R.tc(und)[0]
    dirg = gg.rmat(11, 8, seed=8)  # directed: the formula as it stands
    B = capi.Matrix.from_graph(dirg, np.ones(dirg.nnz, np.int32))
    assert B.triangle_count() == R.tc(dirg)[0]
    # a symmetric graph with self loops (the generator drops loops, so the CSR is built here)
    base = gg.rmat(9, 8, seed=9, undirected=True)
    n = base.n
    rows = np.concatenate([np.repeat(np.arange(n), np.diff(base.row_ptr)), np.arange(0, n, 3)])
    cols = np.concatenate([base.col, np.arange(0, n, 3)])
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    loops = gg.Graph(n=n, row_ptr=np.cumsum(rp).astype(np.int32), col=cols.astype(np.int32))
    Lm = capi.Matrix.from_graph(loops, np.ones(loops.nnz, np.int32))
    assert Lm.triangle_count() == R.tc(loops)[0]
