"""GPU parity of the algorithms run through the lablas:: API on libgbk.

Bit-exact against the oracle and against the reference's own outputs
(tests/golden/) for BFS levels, CC labels, SSSP distances and triangle
counts; PageRank within REL_L1_TOL of the FP64 oracle restatement.
"""
import numpy as np
import pytest

from conftest import REL_L1_TOL, golden_graph, rel_l1
from gb_kun_b200 import graphgen as gg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lc():
    from gb_kun_b200 import lablas_capi
    return lablas_capi


GRAPHS = [
    ("rmat12u", lambda: gg.rmat(12, 16, seed=5, undirected=True)),
    ("er12u", lambda: gg.uniform(12, 8, seed=6, undirected=True)),
    ("rmat11d", lambda: gg.rmat(11, 16, seed=7)),
]


@pytest.mark.parametrize("name,make", GRAPHS)
def test_bfs_vs_oracle(lc, oracle, name, make):
    g = make()
    G = lc.Graph(g)
    for s in gg.sources(g, 4, seed=11):
        lv, _ = G.bfs(int(s))
        assert np.array_equal(lv, oracle.bfs(g, int(s))), (name, s)


@pytest.mark.parametrize("name", ["rmat11u", "er11u", "rmat10"])
def test_bfs_vs_reference_golden(lc, golden, name):
    data, _ = golden
    g = golden_graph(data, name)
    G = lc.Graph(g)
    for k, s in enumerate(data[f"{name}.sources"]):
        lv, _ = G.bfs(int(s))
        assert np.array_equal(lv, data[f"{name}.bfs.{k}"])


@pytest.mark.parametrize("name,make", GRAPHS[:2])
def test_cc_vs_oracle(lc, oracle, name, make):
    g = make()
    lab, _ = lc.Graph(g).cc()
    assert np.array_equal(lab, oracle.cc(g))


@pytest.mark.parametrize("name", ["rmat11u", "er11u"])
def test_cc_vs_reference_golden(lc, golden, name):
    data, _ = golden
    g = golden_graph(data, name)
    lab, _ = lc.Graph(g).cc()
    assert np.array_equal(lab, data[f"{name}.cc"])


@pytest.mark.parametrize("name,make", GRAPHS[:2])
def test_sssp_vs_oracle(lc, oracle, name, make):
    g = make()
    w = gg.weights_i32(g, seed=3)
    G = lc.Graph(g, weights=w)
    inf32 = np.iinfo(np.int32).max
    for s in gg.sources(g, 2, seed=12):
        d = oracle.sssp(g, w, int(s))
        df, _ = G.sssp_f32(int(s))
        di, _ = G.sssp_i32(int(s))
        expect_f = np.where(d < 0, np.float32(np.finfo(np.float32).max), d.astype(np.float32))
        assert np.array_equal(df, expect_f)
        assert np.array_equal(di, np.where(d < 0, inf32, d).astype(np.int32))


@pytest.mark.parametrize("name", ["rmat11u", "er11u"])
def test_sssp_vs_reference_golden(lc, golden, name):
    data, _ = golden
    g = golden_graph(data, name)
    G = lc.Graph(g, weights=data[f"{name}.w"])
    df, _ = G.sssp_f32(int(data[f"{name}.sources"][0]))
    assert np.array_equal(df, data[f"{name}.sssp"])


@pytest.mark.parametrize("name", ["rmat11u", "er11u"])
@pytest.mark.parametrize("iters", [1, 5, 20])
def test_pagerank_vs_reference_golden(lc, oracle, golden, name, iters):
    data, _ = golden
    g = golden_graph(data, name)
    r, it, _ = lc.Graph(g).pagerank(itermax=iters, tol=0.0)
    assert it == iters
    assert rel_l1(r, data[f"{name}.pr.{iters}"]) < REL_L1_TOL
    r64, _, _ = oracle.pagerank(g, tol=0.0, itermax=iters)
    assert rel_l1(r, r64) < REL_L1_TOL


def test_pagerank_tolerance_stop(lc, oracle):
    g = gg.uniform(12, 8, seed=9, undirected=True)  # no sinks: converges
    r64, it64, _ = oracle.pagerank(g, tol=1e-6, itermax=100)
    r, it, _ = lc.Graph(g).pagerank(itermax=100, tol=1e-6)
    assert abs(it - it64) <= 1
    assert rel_l1(r, r64) < REL_L1_TOL


@pytest.mark.parametrize("name,make", GRAPHS[:2])
def test_tc_vs_oracle(lc, oracle, name, make):
    g = make()
    t, _ = lc.Graph(g).tc()
    assert t == oracle.tc(g)


@pytest.mark.parametrize("name", ["rmat11u", "er11u"])
def test_tc_vs_reference_golden(lc, golden, name):
    data, _ = golden
    g = golden_graph(data, name)
    t, _ = lc.Graph(g).tc()
    assert t == int(data[f"{name}.tc"][0])


@pytest.mark.parametrize("fmt", [0])
def test_lablas_spmv_vs_fp64(lc, oracle, fmt):
    g = gg.rmat(12, 16, seed=13)
    val = gg.values_f32(g, seed=1)
    x = gg.vector_f32(g.n, seed=2)
    y, _ = lc.Graph(g).spmv(val, x, fmt=fmt)
    assert rel_l1(y, oracle.spmv_f64(g, val, x)) < REL_L1_TOL


@pytest.mark.parametrize("name,make", GRAPHS)
def test_personalized_pagerank_vs_oracle(lc, oracle, name, make):
    g = make()
    G = lc.Graph(g)
    for s in gg.sources(g, 3, seed=13):
        r, it, _ = G.ppr(int(s), itermax=100, tol=1e-6)
        want, _ = oracle.ppr(g, int(s), damping=0.85, tol=1e-6, itermax=100)
        assert rel_l1(r, want) < REL_L1_TOL, (name, s)
        r7, it7, _ = G.ppr(int(s), itermax=7, tol=0.0)
        want7, _ = oracle.ppr(g, int(s), tol=0.0, itermax=7)
        assert it7 == 7 and rel_l1(r7, want7) < REL_L1_TOL
