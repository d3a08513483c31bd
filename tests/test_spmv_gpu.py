"""GPU parity of gbk_mxv (CSR merge-path SpMV) against the CPU oracle.

Integer / min / or semirings must match bit for bit; FP32 plus-times must be
within REL_L1_TOL (relative L1) of the FP64 oracle.
"""
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


def graphs():
    yield gg.rmat(10, 16, seed=1)
    yield gg.rmat(13, 16, seed=2)
    yield gg.uniform(12, 8, seed=3, undirected=True)
    # one hub row spanning many tiles + empty rows around it
    n = 9000
    src = np.concatenate([np.zeros(8000, np.int64), np.arange(1, 50), [n - 1]])
    dst = np.concatenate([np.arange(1, 8001), np.zeros(49, np.int64), [5]])
    yield gg.from_edges(n, src, dst)
    yield gg.from_edges(5, np.array([], np.int64), np.array([], np.int64))  # no edges at all
    yield gg.from_edges(1, np.array([], np.int64), np.array([], np.int64))  # single vertex


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


KERNELS = [1, 2, 3]  # merge-path tiles, degree bins, runs of 256 entries per warp


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("gi", range(6))
def test_plus_times_f32_vs_fp64(capi, oracle, gi, kernel):
    g = list(graphs())[gi]
    val = gg.values_f32(g, seed=7)
    x = gg.vector_f32(g.n, seed=8)
    A = capi.Matrix.from_graph(g, val)
    A.set_format("CSR", csr_kernel=kernel)
    y = torch.full((g.n,), 7.0, device="cuda")
    A.mxv(dev(x), y)
    ref = oracle.spmv_f64(g, val, x)
    got = y.cpu().numpy()
    assert rel_l1(got, ref) < REL_L1_TOL
    assert np.all(got[g.degrees() == 0] == 0)


SEMIRINGS_EXACT = ["lor_land", "min_plus", "min_second", "min_noteq", "first_min", "structural_bool",
                   "first_wins", "custom_less_plus"]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("sr", SEMIRINGS_EXACT + ["plus_one"])
@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_semirings_exact(capi, oracle, sr, dtype, kernel):
    for g in list(graphs())[:4]:
        if dtype == "f32":
            val = gg.values_f32(g, seed=11)
            x = gg.vector_f32(g.n, seed=12)
            x[::7] = 0
        else:
            val = gg.weights_i32(g, seed=11, lo=0, hi=9)
            x = (gg.vector_f32(g.n, seed=12) * 50).astype(np.int32)
            x[::5] = np.iinfo(np.int32).max
        A = capi.Matrix.from_graph(g, val)
        A.set_format("CSR", csr_kernel=kernel)
        y0 = np.ones(g.n, val.dtype)
        y = dev(y0)
        A.mxv(dev(x), y, semiring=sr)
        expect = oracle.mxv(sr, g, val, x, y0)
        assert np.array_equal(y.cpu().numpy(), expect), (sr, g.name)


@pytest.mark.parametrize("accum", ["plus", "min", "max", "minus", "first", "times"])
def test_accumulators(capi, oracle, accum):
    from gb_kun_b200.capi import BINOP
    g = gg.rmat(11, 8, seed=21)
    val = gg.weights_i32(g, seed=1, lo=1, hi=20)
    x = (gg.vector_f32(g.n, seed=2) * 100).astype(np.int32)
    y0 = (gg.vector_f32(g.n, seed=3) * 1000).astype(np.int32)
    A = capi.Matrix.from_graph(g, val)
    y = dev(y0)
    A.mxv(dev(x), y, semiring="plus_times", accum=accum)
    expect = oracle.mxv("plus_times", g, val, x, y0, accum=BINOP[accum])
    assert np.array_equal(y.cpu().numpy(), expect)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("mode", ["default", "structure", "str_comp", "comp", "scmp"])
@pytest.mark.parametrize("mdtype", ["bool", "f32", "i64"])
def test_dense_mask(capi, oracle, mode, mdtype, kernel):
    from gb_kun_b200.capi import MASK
    g = gg.rmat(12, 8, seed=31, undirected=True)
    val = np.ones(g.nnz, np.float32)
    x = (gg.vector_f32(g.n, seed=4) > 0.7).astype(np.float32)
    m = gg.vector_f32(g.n, seed=5) > 0.5
    mask = {"bool": m.astype(np.bool_), "f32": m.astype(np.float32), "i64": m.astype(np.int64)}[mdtype]
    y0 = np.full(g.n, 3.0, np.float32)
    A = capi.Matrix.from_graph(g, val)
    A.set_format("CSR", csr_kernel=kernel)
    y = dev(y0)
    A.mxv(dev(x), y, semiring="lor_land", mask=dev(mask), mask_mode=mode)
    expect = oracle.mxv("lor_land", g, val, x, y0, mask=mask, mask_mode=MASK[mode])
    assert np.array_equal(y.cpu().numpy(), expect)


def test_transpose_uses_csc(capi, oracle):
    g = gg.rmat(12, 16, seed=41)
    val = gg.weights_i32(g, seed=6, lo=1, hi=255)
    x = (gg.vector_f32(g.n, seed=7) * 1000).astype(np.int32)
    cp, row, _ = oracle.transpose(g)
    # values of A^T in CSC order: edges sorted by (col, row)
    rows = np.repeat(np.arange(g.n), g.degrees())
    tval = val[np.lexsort((rows, g.col))]
    from gb_kun_b200.graphgen import Graph
    gt = Graph(n=g.n, row_ptr=cp, col=row)
    A = capi.Matrix.from_graph(g, val)
    y0 = np.zeros(g.n, np.int32)
    y = dev(y0)
    A.mxv(dev(x), y, semiring="min_plus", transpose=True)
    expect = oracle.mxv("min_plus", gt, tval, x, y0)
    assert np.array_equal(y.cpu().numpy(), expect)
    assert A.info().has_csc == 1


def test_alias_x_is_y(capi, oracle):
    g = gg.rmat(11, 16, seed=51)
    val = gg.values_f32(g, seed=1)
    x = gg.vector_f32(g.n, seed=2)
    A = capi.Matrix.from_graph(g, val)
    xy = dev(x)
    A.mxv(xy, xy, semiring="plus_times", accum="plus")
    expect = x.astype(np.float64) + oracle.spmv_f64(g, val, x)
    assert rel_l1(xy.cpu().numpy(), expect) < REL_L1_TOL


def test_errors_are_reported(capi):
    g = gg.rmat(8, 4, seed=1)
    A = capi.Matrix.from_graph(g, np.ones(g.nnz, np.float32))
    x = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    with pytest.raises(capi.GbkError) as e:
        A.mxv(x, x)
    assert e.value.status == 7  # GBK_DOMAIN_MISMATCH (matrix f32, vectors i32)


@pytest.mark.parametrize("kernel", KERNELS)
def test_repeatable(capi, kernel):
    """Results do not depend on scheduling: two runs are identical."""
    g = gg.rmat(14, 16, seed=61)
    val = gg.values_f32(g, seed=1)
    x = dev(gg.vector_f32(g.n, seed=2))
    A = capi.Matrix.from_graph(g, val)
    A.set_format("CSR", csr_kernel=kernel)
    y1 = torch.empty(g.n, device="cuda")
    y2 = torch.empty(g.n, device="cuda")
    A.mxv(x, y1)
    A.mxv(x, y2)
    assert torch.equal(y1, y2)


def _graph_from_lengths(lengths, seed):
    """Rows of the given lengths, columns drawn without repeats per row."""
    from gb_kun_b200.graphgen import Graph
    lengths = np.asarray(lengths, np.int64)
    n = max(len(lengths), int(lengths.max()) + 1 if len(lengths) else 1)
    lengths = np.concatenate([lengths, np.zeros(n - len(lengths), np.int64)])
    rng = np.random.default_rng(seed)
    ptr = np.zeros(n + 1, np.int32)
    ptr[1:] = np.cumsum(lengths)
    col = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) for k in lengths if k > 0]
                         or [np.zeros(0, np.int64)]).astype(np.int32)
    return Graph(n=n, row_ptr=ptr, col=col)


# Row lengths around the entry-chunk kernel's boundaries (256 entries per
# warp, 8 per lane): rows ending exactly on a chunk / lane edge, rows spanning
# many chunks (over 32: summed by a warp), chunks of more than 32 rows (row
# search over several windows), empty rows between and at both ends, a last
# chunk of 1..255.
CHUNK_CASES = {
    "aligned": [256, 256, 8, 248, 512],
    "straddle": [0, 255, 2, 0, 0, 1, 300, 7, 9, 1, 0, 3000, 1, 1],
    "empty_edges": [0, 0, 0, 17, 0, 1, 0, 2000, 0, 0],
    "ragged_tail": [5] * 61 + [1],
    "one_hub": [4099],
    "two_hubs": [9000, 1, 8193, 8192, 8449],
    "many_rows": [1] * 700 + [0] * 300 + [2] * 200,
    "lane_edges": [8, 16, 7, 1, 9, 15, 24, 1, 255, 1, 257],
}


@pytest.mark.parametrize("case", sorted(CHUNK_CASES))
@pytest.mark.parametrize("sr,dtype", [("plus_times", "f32"), ("min_plus", "i32"), ("lor_land", "f32")])
def test_entry_chunks_row_boundaries(capi, oracle, case, sr, dtype):
    g = _graph_from_lengths(CHUNK_CASES[case], seed=len(case))
    if dtype == "f32":
        val = gg.values_f32(g, seed=3) if g.nnz else np.zeros(0, np.float32)
        x = gg.vector_f32(g.n, seed=4)
    else:
        val = gg.weights_i32(g, seed=3, lo=0, hi=50) if g.nnz else np.zeros(0, np.int32)
        x = (gg.vector_f32(g.n, seed=4) * 100).astype(np.int32)
    A = capi.Matrix.from_graph(g, val)
    A.set_format("CSR", csr_kernel=3)
    y0 = np.full(g.n, 2, val.dtype)
    y = dev(y0)
    A.mxv(dev(x), y, semiring=sr, accum="plus")
    from gb_kun_b200.capi import BINOP
    if sr == "plus_times":
        expect = y0.astype(np.float64) + oracle.spmv_f64(g, val, x)
        assert rel_l1(y.cpu().numpy(), expect) < REL_L1_TOL
    else:
        expect = oracle.mxv(sr, g, val, x, y0, accum=BINOP["plus"])
        assert np.array_equal(y.cpu().numpy(), expect)
    # the same rows under a mask, no accumulator
    m = (np.arange(g.n) % 3) != 1
    y = dev(y0)
    A.mxv(dev(x), y, semiring=sr, mask=dev(m))
    expect = oracle.mxv(sr, g, val, x, y0, mask=m)
    if sr == "plus_times":
        got = y.cpu().numpy()
        assert np.all(got[~m] == 0)
        ref = oracle.spmv_f64(g, val, x)
        assert rel_l1(got[m], ref[m]) < REL_L1_TOL
    else:
        assert np.array_equal(y.cpu().numpy(), expect)
