"""GPU parity at the workload sizes the benchmarks run.

* Plain SpMV: FP32 plus-times on CSR over R-MAT scale 18 (262,144 vertices,
  edge factor 16), against the FP64 oracle and against the reference's own
  CPU CSR SpMV (oracle/_ref) on the same inputs.
* Format sweep: R-MAT and Erdos-Renyi scale 22 (4,194,304 vertices, mean
  degree 16) in every storage format, plus-times FP32 against FP64 and or-and
  bit-exact against the oracle.
* Full algorithms on undirected R-MAT scale 20 (1,048,576 vertices): BFS, CC
  and integer-weight SSSP bit-exact against the reference's own CPU code,
  PageRank within REL_L1_TOL of the FP64 oracle and of the reference; triangle
  counts exact against the reference at scale 18 (its hash-based counter
  takes tens of seconds beyond that) and against the oracle at scale 20.
* Batched traversals on R-MAT scale 22: every one of 64 BFS lanes bit-exact
  and every one of 32 PPR lanes within REL_L1_TOL of the FP64 oracle.

The checkers run on the host; independent oracle calls run on a thread pool
(the ctypes calls release the GIL).
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import REL_L1_TOL, rel_l1
from gb_kun_b200 import graphgen as gg

pytestmark = pytest.mark.gpu

INF32 = np.iinfo(np.int32).max


@pytest.fixture(scope="module")
def torch():
    import torch as t
    from gb_kun_b200 import capi
    capi.init(0)
    return t


@pytest.fixture(scope="module")
def ref():
    from oracle.cpu import Reference
    if not Reference.available():
        pytest.skip("reference CPU library not built (oracle/_ref)")
    return Reference()


def _pool():
    import os
    return ThreadPoolExecutor(max_workers=max(2, min(16, os.cpu_count() or 2)))


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _written_rows(g):
    """Rows the reference CSR SpMV writes: it skips the trailing empty rows
    when nnz is a multiple of its thread count (balancing.h:12-22)."""
    deg = np.diff(g.row_ptr)
    nz = np.nonzero(deg)[0]
    last = int(nz[-1]) + 1 if len(nz) else 0
    keep = np.zeros(g.n, bool)
    keep[:last] = True
    return keep


# ---- plain SpMV: R-MAT scale 18, CSR -------------------------------------

@pytest.fixture(scope="module")
def rmat18():
    g = gg.rmat(18, 16, seed=42)
    return g, gg.values_f32(g, seed=43), gg.vector_f32(g.n, seed=44)


@pytest.mark.parametrize("kernel", [1, 2, 3], ids=["merge", "bins", "chunks"])
def test_csr_s18_vs_fp64_and_reference(torch, oracle, ref, rmat18, kernel):
    from gb_kun_b200 import capi
    g, val, x = rmat18
    assert g.n == 262144 and g.nnz > 3_500_000
    A = capi.Matrix.from_graph(g, val)
    A.set_format("CSR", csr_kernel=kernel)
    y = torch.zeros(g.n, device="cuda")
    A.mxv(_dev(torch, x), y)
    got = y.cpu().numpy()
    assert rel_l1(got, oracle.spmv_f64(g, val, x)) < REL_L1_TOL
    want, _ = ref.spmv(g, val, x, fmt=0)  # the reference's CSR GrB_mxv
    keep = _written_rows(g)
    assert rel_l1(got[keep], want[keep]) < REL_L1_TOL
    A.close()


# ---- format sweep: R-MAT and Erdos-Renyi scale 22 -------------------------

SWEEP = [
    ("CSR_bins", dict(fmt="CSR", csr_kernel=2)),
    ("CSR_merge", dict(fmt="CSR", csr_kernel=1)),
    ("CSR_chunks", dict(fmt="CSR", csr_kernel=3)),
    ("SELL_C_s1", dict(fmt="SELL_C", sigma=1)),
    ("SELL_C_s256", dict(fmt="SELL_C", sigma=256)),
    ("SELL_C_s4096", dict(fmt="SELL_C", sigma=4096)),
    ("SELL_C_s4096_reorder", dict(fmt="SELL_C", sigma=4096, reorder_cols=1)),
    ("SELL_C_staged", dict(fmt="SELL_C", seg_staged=1)),
    ("SELL_C_staged_reorder", dict(fmt="SELL_C", seg_staged=1, reorder_cols=1)),
    ("CSR_SEG", dict(fmt="CSR_SEG")),
    ("CSR_SEG_merge", dict(fmt="CSR_SEG", seg_staged=-1)),
    ("LAV", dict(fmt="LAV")),
]


@pytest.fixture(scope="module", params=["rmat22", "er22"])
def graph22(request, oracle):
    name = request.param
    g = gg.rmat(22, 16, seed=42) if name == "rmat22" else gg.uniform(22, 16, seed=42)
    val = gg.values_f32(g, seed=43)
    x = gg.vector_f32(g.n, seed=44)
    wi = np.ones(g.nnz, np.int32)
    xb = (gg.vector_f32(g.n, seed=45) < 0.05).astype(np.int32)
    y0 = np.zeros(g.n, np.int32)
    return {"name": name, "g": g, "val": val, "x": x, "ref64": oracle.spmv_f64(g, val, x), "wi": wi, "xb": xb,
            "or_and": oracle.mxv("lor_land", g, wi, xb, y0)}


@pytest.mark.parametrize("label,fmt", SWEEP, ids=[s[0] for s in SWEEP])
def test_format_sweep_s22(torch, graph22, label, fmt):
    from gb_kun_b200 import capi
    d = graph22
    g = d["g"]
    assert g.n == 4194304
    f = dict(fmt)
    name = f.pop("fmt")
    A = capi.Matrix.from_graph(g, d["val"])
    A.set_format(name, **f)
    y = torch.zeros(g.n, device="cuda")
    A.mxv(_dev(torch, d["x"]), y)
    err = rel_l1(y.cpu().numpy(), d["ref64"])
    assert err < REL_L1_TOL, (d["name"], label, err)
    A.close()
    B = capi.Matrix.from_graph(g, d["wi"])
    B.set_format(name, **f)
    yb = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    B.mxv(_dev(torch, d["xb"]), yb, semiring="lor_land")
    assert np.array_equal(yb.cpu().numpy(), d["or_and"]), (d["name"], label)
    B.close()


# ---- full algorithms: undirected R-MAT scale 20 ---------------------------

@pytest.fixture(scope="module")
def alg20():
    from gb_kun_b200 import lablas_capi as lc
    g = gg.rmat(20, 16, seed=42, undirected=True)
    w = gg.weights_i32(g, seed=45)
    G = lc.Graph(g, weights=w)
    return g, w, G


def test_bfs_s20_vs_reference(alg20, ref):
    g, _, G = alg20
    for s in gg.sources(g, 3, seed=46):
        lv, _ = G.bfs(int(s))
        want, _ = ref.bfs(g, int(s))
        assert np.array_equal(lv, want), int(s)


def test_cc_s20_vs_reference(alg20, ref):
    g, _, G = alg20
    lab, _ = G.cc()
    want, _ = ref.cc(g)
    assert np.array_equal(lab, want)


def test_sssp_s20_vs_reference(alg20, ref, oracle):
    g, w, G = alg20
    for s in gg.sources(g, 2, seed=47):
        df, _ = G.sssp_f32(int(s))
        want, _ = ref.sssp(g, w, int(s))  # float weights carrying exact integers
        assert np.array_equal(df, want), int(s)
        di, _ = G.sssp_i32(int(s))
        d64 = oracle.sssp(g, w, int(s))
        assert np.array_equal(di, np.where(d64 < 0, INF32, d64).astype(np.int32))


def test_pagerank_s20_vs_fp64_and_reference(alg20, ref, oracle):
    g, _, G = alg20
    r, it, _ = G.pagerank(itermax=100, damping=0.85, tol=1e-6)
    r64, _, _ = oracle.pagerank(g, tol=0.0, itermax=it)
    assert rel_l1(r, r64) < REL_L1_TOL
    rr, _ = ref.pagerank(g, it)
    # the reference accumulates in FP32 in another order; its own distance
    # from FP64 bounds how close the two FP32 results can be
    ref_err = rel_l1(rr, r64)
    assert rel_l1(r, rr) < max(REL_L1_TOL, 2 * ref_err)


def test_tc_s20_vs_oracle(alg20, oracle):
    g, _, G = alg20
    t, _ = G.tc()
    assert t == oracle.tc(g)


def test_tc_s18_vs_reference(ref):
    from gb_kun_b200 import lablas_capi as lc
    g = gg.rmat(18, 16, seed=42, undirected=True)
    t, _ = lc.Graph(g).tc()
    want, _ = ref.tc(g)
    assert t == want


# ---- batched traversals: R-MAT scale 22, every lane -----------------------

@pytest.fixture(scope="module")
def batch22():
    from gb_kun_b200 import capi
    g = gg.rmat(22, 16, seed=42)
    A = capi.Matrix.from_graph(g, val=gg.weights_i32(g, seed=45).astype(np.float32))
    yield g, A
    A.close()


def test_msbfs64_s22_every_lane(torch, oracle, batch22):
    g, A = batch22
    src = gg.sources(g, 64, seed=46).astype(np.int32)
    assert len(src) == 64
    lv = torch.zeros((64, g.n), dtype=torch.int32, device="cuda")
    A.msbfs(src, lv)
    got = lv.cpu().numpy()
    with _pool() as ex:
        want = list(ex.map(lambda s: oracle.bfs(g, int(s)), src))
    for k in range(64):
        assert np.array_equal(got[k], want[k]), (k, int(src[k]))


def test_ppr32_s22_every_lane(torch, oracle, batch22):
    g, A = batch22
    src = gg.sources(g, 32, seed=47).astype(np.int32)
    r = torch.zeros((32, g.n), dtype=torch.float32, device="cuda")
    A.ppr(src, r, damping=0.85, tol=1e-6, itermax=100)
    got = r.cpu().numpy()
    with _pool() as ex:
        want = list(ex.map(lambda s: oracle.ppr(g, int(s), damping=0.85, tol=1e-6, itermax=100)[0], src))
    for k in range(32):
        err = rel_l1(got[k], want[k])
        assert err < REL_L1_TOL, (k, int(src[k]), err)
