"""GPU parity of the optimised storage formats (SELL-C-sigma, CSR_SEG, LAV)
against the oracle, in both orientations (mxv over A, vxm over A^T)."""
import numpy as np
import pytest

from conftest import REL_L1_TOL, rel_l1
from gb_kun_b200 import graphgen as gg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def capi():
    from gb_kun_b200 import capi
    capi.init(0)
    return capi


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def hub_graph():
    n = 20000
    src = np.concatenate([np.zeros(15000, np.int64), np.full(3000, 7), np.arange(100, 400)])
    dst = np.concatenate([np.arange(1, 15001), np.arange(2000, 5000), np.full(300, 3)])
    return gg.from_edges(n, src, dst)


GRAPHS = {
    "rmat13": lambda: gg.rmat(13, 16, seed=3),
    "er12": lambda: gg.uniform(12, 8, seed=4),
    "rmat12u": lambda: gg.rmat(12, 16, seed=5, undirected=True),
    "hub": hub_graph,
}

FORMATS = [("SELL_C", 1), ("SELL_C", 256), ("SELL_C", 4096), ("SELL_C_HOT", 4096), ("SELL_C_HOT", 1), ("CSR_SEG", 0),
           ("CSR_SEG_MERGE", 0), ("LAV", 0), ("SELL_C_STAGED", 0), ("SELL_C_STAGED", 1)]


def apply(A, fmt, sigma, seg_cols):
    """SELL_C_HOT: SELL-C with 1024 shared-memory x columns; CSR_SEG is the
    staged-window kernel, CSR_SEG_MERGE the unstaged segments with a merge."""
    if fmt == "SELL_C_HOT":
        A.set_format("SELL_C", sigma=sigma, hot_cols=1024)
    elif fmt == "SELL_C_STAGED":
        A.set_format("SELL_C", seg_staged=1, reorder_cols=sigma)  # sigma column: 1 = renumber columns
    elif fmt == "CSR_SEG_MERGE":
        A.set_format("CSR_SEG", seg_cols=seg_cols, seg_staged=-1)
    else:
        A.set_format(fmt, sigma=sigma, seg_cols=seg_cols if fmt != "SELL_C" else 0)


def transposed(oracle, g, val):
    cp, row, _ = oracle.transpose(g)
    rows = np.repeat(np.arange(g.n), g.degrees())
    return gg.Graph(n=g.n, row_ptr=cp, col=row), val[np.lexsort((rows, g.col))]


@pytest.mark.parametrize("gname", sorted(GRAPHS))
@pytest.mark.parametrize("fmt,sigma", FORMATS)
@pytest.mark.parametrize("transpose", [False, True])
def test_plus_times_f32(capi, oracle, gname, fmt, sigma, transpose):
    g = GRAPHS[gname]()
    val = gg.values_f32(g, seed=1)
    x = gg.vector_f32(g.n, seed=2)
    A = capi.Matrix.from_graph(g, val)
    apply(A, fmt, sigma, 1024)
    y = torch.full((g.n,), 5.0, device="cuda")
    A.mxv(dev(x), y, transpose=transpose, accum="plus")
    go, vo = transposed(oracle, g, val) if transpose else (g, val)
    expect = 5.0 + oracle.spmv_f64(go, vo, x)
    assert rel_l1(y.cpu().numpy(), expect) < REL_L1_TOL


@pytest.mark.parametrize("fmt,sigma", FORMATS)
@pytest.mark.parametrize("sr", ["min_plus", "lor_land", "min_second", "plus_one"])
def test_exact_semirings_i32(capi, oracle, fmt, sigma, sr):
    for gname in ("rmat13", "hub"):
        g = GRAPHS[gname]()
        val = gg.weights_i32(g, seed=3, lo=1, hi=100)
        x = (gg.vector_f32(g.n, seed=4) * 1000).astype(np.int32)
        x[::3] = 0
        A = capi.Matrix.from_graph(g, val)
        apply(A, fmt, sigma, 512)
        for transpose in (False, True):
            y0 = np.full(g.n, 9, np.int32)
            y = dev(y0)
            A.mxv(dev(x), y, semiring=sr, transpose=transpose)
            go, vo = transposed(oracle, g, val) if transpose else (g, val)
            assert np.array_equal(y.cpu().numpy(), oracle.mxv(sr, go, vo, x, y0)), (gname, transpose)


def test_sell_padding_accounting(capi):
    g = gg.rmat(13, 16, seed=3)
    A = capi.Matrix.from_graph(g, gg.values_f32(g))
    A.set_format("SELL_C", sigma=4096)
    padded = A.info().padded_nnz
    assert padded >= g.nnz
    A.set_format("SELL_C", sigma=1)
    assert A.info().padded_nnz >= g.nnz


def test_autotune_picks_a_correct_format_and_caches(capi, oracle):
    g = GRAPHS["rmat13"]()
    val = gg.values_f32(g, seed=7)
    x = gg.vector_f32(g.n, seed=8)
    A = capi.Matrix.from_graph(g, val)
    r1 = A.autotune(reps=3)
    assert r1.cached == 0 and r1.best_ms > 0
    assert all(r1.candidate_ms[i] > 0 for i in range(r1.ncandidates))
    y = torch.zeros(g.n, device="cuda")
    A.mxv(dev(x), y)
    assert rel_l1(y.cpu().numpy(), oracle.spmv_f64(g, val, x)) < REL_L1_TOL
    B = capi.Matrix.from_graph(g, val)  # same graph: the choice comes from the cache
    r2 = B.autotune(reps=3)
    assert r2.cached == 1 and r2.format == r1.format and r2.sell_sigma == r1.sell_sigma
    assert B.info().format == r1.format


def test_masked_call_uses_csr_semantics(capi, oracle):
    """Masked SpMV always runs the CSR kernel, as the reference's SpMV does."""
    g = GRAPHS["rmat12u"]()
    val = np.ones(g.nnz, np.float32)
    A = capi.Matrix.from_graph(g, val)
    A.set_format("LAV")
    x = (gg.vector_f32(g.n, seed=5) > 0.5).astype(np.float32)
    m = (gg.vector_f32(g.n, seed=6) > 0.5).astype(np.float32)
    y0 = np.zeros(g.n, np.float32)
    y = dev(y0)
    A.mxv(dev(x), y, semiring="lor_land", mask=dev(m), mask_mode="str_comp")
    assert np.array_equal(y.cpu().numpy(), oracle.mxv("lor_land", g, val, x, y0, mask=m, mask_mode=5))


@pytest.mark.parametrize("fmt", ["CSR_SEG", "LAV", "SELL_C_STAGED", "SELL_C_STAGED_REORDER"])
@pytest.mark.parametrize("sr", ["plus_times", "min_plus", "lor_land", "plus_one", "min_second", "first_wins"])
@pytest.mark.parametrize("accum", ["second", "plus"])
def test_staged_segments_many_windows(capi, oracle, fmt, sr, accum):
    """CSR_SEG, LAV (columns renumbered by in-degree on the device) and
    SELL-C-sigma inside windows (columns in their order or renumbered), with
    x windows in shared memory on a graph of 3 windows (131072 columns),
    every add class (atomic add / min / or) and the CSR fallback for a
    non-associative add; float sums within REL_L1_TOL, integers exact."""
    g = gg.rmat(17, 12, seed=8)
    if sr == "plus_times":
        val = gg.values_f32(g, seed=1)
        x = gg.vector_f32(g.n, seed=2)
        y0 = np.full(g.n, 0.5, np.float32)
    else:
        val = gg.weights_i32(g, seed=3, lo=1, hi=100)
        x = (gg.vector_f32(g.n, seed=4) * 1000).astype(np.int32)
        x[::5] = 0
        y0 = np.full(g.n, 7, np.int32)
    A = capi.Matrix.from_graph(g, val)
    if fmt.startswith("SELL_C_STAGED"):
        A.set_format("SELL_C", seg_staged=1, reorder_cols=int(fmt.endswith("REORDER")))
    else:
        A.set_format(fmt)
    for transpose in (False, True):
        y = dev(y0.copy())
        A.mxv(dev(x), y, semiring=sr, accum=accum, transpose=transpose)
        go, vo = transposed(oracle, g, val) if transpose else (g, val)
        acc_code = {"second": 0, "plus": 2}[accum]
        expect = oracle.mxv(sr, go, vo, x, y0.copy(), accum=acc_code)
        got = y.cpu().numpy()
        if sr == "plus_times":
            assert rel_l1(got, expect) < REL_L1_TOL, (transpose, rel_l1(got, expect))
        else:
            assert np.array_equal(got, expect), (sr, accum, transpose)


def test_lav_renumbering_matches_reference_order(capi, oracle):
    """The device LAV build orders columns by in-degree, descending, ties in
    column order (lav/build.hpp:113-141): the result must not depend on it,
    but the staged and the unstaged LAV (both renumbered) must agree exactly
    on an integer semiring, and both with the oracle."""
    g = gg.rmat(16, 16, seed=9)
    val = gg.weights_i32(g, seed=3, lo=1, hi=100)
    x = (gg.vector_f32(g.n, seed=4) * 1000).astype(np.int32)
    y0 = np.zeros(g.n, np.int32)
    want = oracle.mxv("min_plus", g, val, x, y0)
    A = capi.Matrix.from_graph(g, val)
    outs = []
    for staged in (0, -1):
        A.set_format("LAV", seg_staged=staged)
        y = dev(y0.copy())
        A.mxv(dev(x), y, semiring="min_plus")
        outs.append(y.cpu().numpy())
    assert np.array_equal(outs[0], want) and np.array_equal(outs[1], want)


def test_staged_sell_long_rows_and_pieces(capi, oracle):
    """Staged SELL-C on a hub graph: virtual rows longer than 32 entries are
    cut into pieces, every piece folds into its row; plus-times within
    REL_L1_TOL, min-plus exact; accumulate into a non-zero y."""
    g = hub_graph()
    for reorder in (0, 1):
        val = gg.values_f32(g, seed=5)
        x = gg.vector_f32(g.n, seed=6)
        A = capi.Matrix.from_graph(g, val)
        A.set_format("SELL_C", seg_staged=1, reorder_cols=reorder)
        assert A.info().padded_nnz >= g.nnz
        y = dev(np.full(g.n, 0.25, np.float32))
        A.mxv(dev(x), y, accum="plus")
        assert rel_l1(y.cpu().numpy(), 0.25 + oracle.spmv_f64(g, val, x)) < REL_L1_TOL
        vi = gg.weights_i32(g, seed=7, lo=1, hi=90)
        xi = (gg.vector_f32(g.n, seed=8) * 500).astype(np.int32)
        B = capi.Matrix.from_graph(g, vi)
        B.set_format("SELL_C", seg_staged=1, reorder_cols=reorder)
        y0 = np.full(g.n, 3, np.int32)
        yi = dev(y0.copy())
        B.mxv(dev(xi), yi, semiring="min_plus", accum="min")
        assert np.array_equal(yi.cpu().numpy(), oracle.mxv("min_plus", g, vi, xi, y0, accum=6))
