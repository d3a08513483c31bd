"""GPU checks of the element-wise, conversion, reduction, SpMSpV and SpGEMM
entry points of the C ABI against the reference semantics (restated here
in numpy / by the C oracle), including the reference's mask quirks."""
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


def rng(seed=0):
    return np.random.default_rng(seed)


def test_sparse_dense_round_trip(capi):
    for n, dens in [(0, 0.0), (1, 1.0), (1000, 0.0), (5000, 0.01), (100000, 0.3), (70000, 1.0)]:
        r = rng(n)
        x = np.where(r.random(n) < dens, r.random(n).astype(np.float32) + 0.5, 0).astype(np.float32)
        ids, vals = capi.to_sparse(dev(x))
        nz = np.nonzero(x)[0]
        assert np.array_equal(ids.cpu().numpy(), nz.astype(np.int32))
        assert np.array_equal(vals.cpu().numpy(), x[nz])
        if n:
            assert np.array_equal(capi.to_dense(ids, vals, n).cpu().numpy(), x)
            assert capi.nvals(dev(x)) == len(nz)


@pytest.mark.parametrize("op,expect", [("plus", lambda a, b: a + b), ("min", np.minimum),
                                       ("lt", lambda a, b: (a < b)), ("ne", lambda a, b: a != b),
                                       ("div", lambda a, b: a / b)])
@pytest.mark.parametrize("mask_kind", ["none", "dense", "sparse"])
def test_ewise(capi, op, expect, mask_kind):
    n = 4097
    r = rng(1)
    u = r.random(n).astype(np.float32)
    v = r.random(n).astype(np.float32) + 0.1
    w0 = np.full(n, -1.0, np.float32)
    w = dev(w0)
    m = r.random(n) < 0.4
    mask = None
    sel = np.ones(n, bool)
    if mask_kind == "dense":
        mask = capi.dense_mask(dev(m.astype(np.uint8).view(np.bool_)))
        sel = m
    elif mask_kind == "sparse":
        ids = dev(np.nonzero(m)[0].astype(np.int32))
        mask = capi.sparse_mask(ids, mode="str_comp")  # the mode is not consulted by element-wise ops
        sel = m
        keep = ids
    capi.ewise(op, capi.F32, w, dev(u), dev(v), mask=mask)
    exp = w0.copy()
    exp[sel] = expect(u, v)[sel].astype(np.float32)
    assert np.array_equal(w.cpu().numpy(), exp)


def test_ewise_mixed_types(capi):
    n = 1000
    r = rng(2)
    a = r.integers(0, 5, n).astype(np.int32)
    b = r.integers(0, 5, n).astype(np.int32)
    w = torch.zeros(n, dtype=torch.bool, device="cuda")
    capi.ewise("ne", capi.I32, w, dev(a), dev(b))
    assert np.array_equal(w.cpu().numpy(), a != b)


@pytest.mark.parametrize("mode", ["default", "structure", "str_comp", "comp", "scmp"])
@pytest.mark.parametrize("form", ["dense", "sparse"])
def test_assign_scalar_modes(capi, mode, form):
    n = 3000
    r = rng(3)
    m = r.random(n) < 0.3
    w0 = r.random(n).astype(np.float32)
    w = dev(w0)
    if form == "dense":
        mask = capi.dense_mask(dev(m.astype(np.float32)), mode)
    else:
        mask = capi.sparse_mask(dev(np.nonzero(m)[0].astype(np.int32)), mode)
    capi.assign_scalar(w, 7.0, mask=mask)
    exp = w0.copy()
    if mode in ("default", "structure"):
        exp[m] = 7.0
    elif mode == "str_comp":
        exp[~m] = 7.0
    assert np.array_equal(w.cpu().numpy(), exp)  # COMP / SCMP assign nothing (generic_operations.h:52-59)


def test_assign_vector_sparse_mask_reads_list_position(capi):
    """assign(w, sparse mask, u): w[ids[k]] = u[k] (generic_operations.h:28-34)."""
    n = 2000
    r = rng(4)
    u = r.random(n).astype(np.float32)
    ids = np.sort(r.choice(n, 300, replace=False)).astype(np.int32)
    w0 = np.zeros(n, np.float32)
    w = dev(w0)
    capi.assign_vector("second", capi.F32, w, dev(u), mask=capi.sparse_mask(dev(ids), "structure"))
    exp = w0.copy()
    exp[ids] = u[:len(ids)]
    assert np.array_equal(w.cpu().numpy(), exp)
    # dense mask form: w[i] = u[i]
    w = dev(w0)
    m = np.zeros(n, np.float32)
    m[ids] = 1
    capi.assign_vector("second", capi.F32, w, dev(u), mask=capi.dense_mask(dev(m), "structure"))
    exp = w0.copy()
    exp[ids] = u[ids]
    assert np.array_equal(w.cpu().numpy(), exp)


def test_assign_scatter_repeated_indices_take_last(capi):
    """w[idx[k]] = u[k]; a repeated index keeps the value of its largest k."""
    n = 2000
    r = rng(5)
    idx = r.integers(0, 50, n).astype(np.int32)
    u = np.arange(n, dtype=np.int32)
    w = dev(np.full(n, -5, np.int32))
    capi.assign_vector("second", capi.I32, w, dev(u), indices=dev(idx))
    exp = np.full(n, -5, np.int32)
    for k, i in enumerate(idx):
        exp[i] = u[k]
    assert np.array_equal(w.cpu().numpy(), exp)


def test_extract_gather_and_sparse_quirk(capi):
    n = 3000
    r = rng(6)
    u = r.integers(0, 1000, n).astype(np.int32)
    idx = r.integers(0, n, n).astype(np.int32)
    w = dev(np.zeros(n, np.int32))
    capi.extract("second", capi.I32, w, dev(u), indices=dev(idx))
    assert np.array_equal(w.cpu().numpy(), u[idx])
    ids = np.sort(r.choice(n, 100, replace=False)).astype(np.int32)
    w0 = np.zeros(n, np.int32)
    w = dev(w0)
    capi.extract("second", capi.I32, w, dev(u), mask=capi.sparse_mask(dev(ids)))
    exp = w0.copy()
    exp[:len(ids)] = u[ids]  # w[k] = u[ids[k]] (generic_operations.h:85-92)
    assert np.array_equal(w.cpu().numpy(), exp)


def test_reduce(capi):
    r = rng(7)
    x = r.random(1_000_003).astype(np.float32)
    assert abs(capi.reduce("plus", capi.F64, dev(x)) - x.astype(np.float64).sum()) < 1e-6 * x.size
    i = r.integers(-1000, 1000, 77777).astype(np.int32)
    assert capi.reduce("min", capi.I32, dev(i)) == i.min()
    assert capi.reduce("max", capi.I32, dev(i)) == i.max()
    assert capi.reduce("plus", capi.I64, dev(i)) == int(i.astype(np.int64).sum())
    b = np.zeros(1000, np.bool_)
    assert capi.reduce("lor", capi.BOOL, dev(b)) == 0
    b[999] = True
    assert capi.reduce("lor", capi.BOOL, dev(b)) == 1
    assert capi.reduce("plus", capi.F32, dev(np.zeros(0, np.float32))) == 0.0


@pytest.mark.parametrize("sr,dtype", [("lor_land", "f32"), ("plus_times", "f32"), ("min_plus", "i32"),
                                      ("min_second", "i32"), ("plus_one", "i32"), ("first_wins", "f32")])
@pytest.mark.parametrize("mask_kind", ["none", "dense", "dense_comp", "sparse_comp"])
@pytest.mark.parametrize("transpose", [False, True])
def test_spmspv_vs_oracle(capi, oracle, sr, dtype, mask_kind, transpose):
    from gb_kun_b200.capi import MASK
    g = gg.rmat(11, 16, seed=21)
    if dtype == "f32":
        val = gg.values_f32(g, seed=1)
    else:
        val = gg.weights_i32(g, seed=1, lo=1, hi=50)
    A = capi.Matrix.from_graph(g, val)
    r = rng(8)
    f_ids = np.sort(r.choice(g.n, 150, replace=False)).astype(np.int32)
    f_vals = (r.random(len(f_ids)) * 10 + 1).astype(val.dtype)
    y0 = (r.random(g.n) * 5).astype(val.dtype)
    m = r.random(g.n) < 0.5
    mask = None
    omask, omode = None, 6
    if mask_kind == "dense":
        mask = capi.dense_mask(dev(m.astype(np.float32)), "default")
        omask, omode = m.astype(np.float32), MASK["default"]
    elif mask_kind == "dense_comp":
        mask = capi.dense_mask(dev(m.astype(np.float32)), "str_comp")
        omask, omode = m.astype(np.float32), MASK["str_comp"]
    elif mask_kind == "sparse_comp":
        mask = capi.sparse_mask(dev(np.nonzero(m)[0].astype(np.int32)), "str_comp")
        omask, omode = m.astype(np.float32), MASK["str_comp"]
    y = dev(y0)
    A.spmspv(dev(f_ids), dev(f_vals), y, semiring=sr, accum="plus", mask=mask, transpose=transpose)
    # oracle pushes along the CSR given to it: vxm (transpose) uses A, mxv uses A^T
    if transpose:
        go, vo = g, val
    else:
        cp, row, _ = oracle.transpose(g)
        rows = np.repeat(np.arange(g.n), g.degrees())
        vo = val[np.lexsort((rows, g.col))]
        go = gg.Graph(n=g.n, row_ptr=cp, col=row)
    expect = oracle.spmspv(sr, go, vo, f_ids, f_vals, y0, accum=2, mask=omask, mask_mode=omode)
    got = y.cpu().numpy()
    if sr == "plus_times":
        assert rel_l1(got, expect) < REL_L1_TOL
    else:
        assert np.array_equal(got, expect)


@pytest.mark.parametrize("mode", ["default", "str_comp"])
def test_mxv_sparse_mask(capi, oracle, mode):
    g = gg.rmat(11, 16, seed=22, undirected=True)
    val = gg.weights_i32(g, seed=2, lo=1, hi=9)
    x = rng(9).integers(0, 100, g.n).astype(np.int32)
    ids = np.sort(rng(10).choice(g.n, 400, replace=False)).astype(np.int32)
    A = capi.Matrix.from_graph(g, val)
    y0 = np.full(g.n, -3, np.int32)
    y = dev(y0)
    A.mxv_sparse_mask(dev(x), y, dev(ids), semiring="plus_times", accum="plus", mask_mode=mode)
    full = oracle.mxv("plus_times", g, val, x, y0, accum=2)
    exp = y0.copy()
    sel = np.zeros(g.n, bool)
    sel[ids] = True
    if mode == "default":
        exp[sel] = full[sel]  # unlisted rows keep y (spmv_csr.h:200-213)
    else:
        exp[~sel] = full[~sel]
        exp[sel] = 0
    assert np.array_equal(y.cpu().numpy(), exp)


def test_mxm_masked_counts(capi, oracle):
    g = gg.rmat(11, 16, seed=23, undirected=True)
    one = np.ones(g.nnz, np.int32)
    A = capi.Matrix.from_graph(g, one)
    Cm = A.mxm_masked(A, A, semiring="plus_one")
    assert Cm.info().nnz == g.nnz
    _, _, v = Cm.arrays()
    import ctypes
    out = ctypes.c_int64()
    capi.check(capi.lib().gbk_reduce(0, capi.I64, ctypes.c_void_p(v), capi.I32, g.nnz, ctypes.byref(out),
                                     capi.stream_ptr()), "gbk_reduce")
    assert out.value == 6 * oracle.tc(g)


@pytest.mark.parametrize("sr,dtype", [("lor_land", "f32"), ("plus_times", "f32"), ("min_plus", "i32"),
                                      ("min_second", "i32"), ("plus_one", "i32"), ("custom_less_plus", "f32")])
@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("nf", [0, 1, 150, 2048])
def test_spmspv_sparse_output_vs_oracle(capi, oracle, sr, dtype, transpose, nf):
    """The map-based sparse-output push (spmspv_maps.h:5-142): every reached row
    once, ids ascending, value = the semiring's add over its products (or 1
    when add probes to 1, as the or-map and a less-monoid do)."""
    g = gg.rmat(11, 16, seed=23)
    val = gg.values_f32(g, seed=1) if dtype == "f32" else gg.weights_i32(g, seed=1, lo=1, hi=50)
    A = capi.Matrix.from_graph(g, val)
    r = rng(11)
    f_ids = np.sort(r.choice(g.n, nf, replace=False)).astype(np.int32)
    f_vals = (r.random(nf) * 10 + 1).astype(val.dtype)
    ids, vals = A.spmspv_sparse(dev(f_ids), dev(f_vals), semiring=sr, transpose=transpose)
    if transpose:
        go, vo = g, val
    else:
        cp, row, _ = oracle.transpose(g)
        rows = np.repeat(np.arange(g.n), g.degrees())
        vo = val[np.lexsort((rows, g.col))]
        go = gg.Graph(n=g.n, row_ptr=cp, col=row)
    reached = np.unique(np.concatenate([go.col[go.row_ptr[i]:go.row_ptr[i + 1]] for i in f_ids])
                        if nf else np.zeros(0, np.int32))
    assert np.array_equal(ids.cpu().numpy(), reached.astype(np.int32))
    got = vals.cpu().numpy()
    if sr in ("lor_land", "custom_less_plus"):
        assert (got == 1).all()
        return
    ident = {"plus_times": 0, "plus_one": 0, "min_plus": np.iinfo(np.int32).max,
             "min_second": np.iinfo(np.int32).max}[sr]
    y0 = np.full(g.n, ident, val.dtype)
    dense = oracle.spmspv(sr, go, vo, f_ids, f_vals, y0)
    if sr == "plus_times":
        assert rel_l1(got, dense[reached]) < REL_L1_TOL
    else:
        assert np.array_equal(got, dense[reached])


def test_spmspv_sparse_output_refuses_a_mask(capi):
    g = gg.rmat(8, 8, seed=24)
    A = capi.Matrix.from_graph(g, gg.values_f32(g))
    ids = dev(np.array([1, 2], np.int32))
    vals = dev(np.ones(2, np.float32))
    m = capi.dense_mask(dev(np.ones(g.n, np.float32)))
    import ctypes as C
    y_ids = torch.empty(g.n, dtype=torch.int32, device="cuda")
    y_vals = torch.empty(g.n, dtype=torch.float32, device="cuda")
    nv = C.c_int64()
    rc = capi.lib().gbk_spmspv_sparse(A.h, 0, capi.SEMIRING["plus_times"], capi.F32, capi.ptr(ids), capi.ptr(vals), 2,
                                      capi.ptr(y_ids), capi.ptr(y_vals), C.byref(nv), C.byref(m), capi.stream_ptr())
    assert rc == 21  # GBK_UNSUPPORTED
