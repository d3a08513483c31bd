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


KERNELS = [1, 2]  # merge-path tiles, degree bins


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


def test_repeatable(capi):
    """Merge-path results do not depend on scheduling: two runs are identical."""
    g = gg.rmat(14, 16, seed=61)
    val = gg.values_f32(g, seed=1)
    x = dev(gg.vector_f32(g.n, seed=2))
    A = capi.Matrix.from_graph(g, val)
    y1 = torch.empty(g.n, device="cuda")
    y2 = torch.empty(g.n, device="cuda")
    A.mxv(x, y1)
    A.mxv(x, y2)
    assert torch.equal(y1, y2)
