"""The reference's own algorithm files, unmodified, on the GPU library.

tests/dropin/_bin/ref_algorithms compiles the reference's algorithms/*.hpp
(bfs, bfs_traditional, cc, cc_traditional, pr, pr_traditional, sssp,
sssp_blast, sssp_traditional, tc) against the drop-in header
gb_kun_b200/dropin/src/gb_kun.h and runs them the way the reference's
drivers do.  Their outputs must equal the reference's own outputs
(tests/golden/, made by the reference's CPU build): BFS levels, CC labels,
SSSP distances and triangle counts bit-exact, PageRank within REL_L1_TOL.
The sequential checkers (*_traditional.hpp) read the host CSR view and
write the host copy of their result vector; BFS, CC and Dijkstra must agree
with the GraphBLAS algorithms as the reference's drivers require, and the
sequential PageRank (its own normalisation) with an FP64 restatement of it.  The Cohen triangle
count needs a select with a C++ lambda (tc.hpp:55-70), which cannot run on
the device: it must be refused with an error, not computed on the host.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REL_L1_TOL, golden_graph, rel_l1
from gb_kun_b200 import graphgen as gg

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "dropin" / "_bin" / "ref_algorithms"


def run(tmp_path, g, w, source, pr_iters):
    if not BIN.exists():
        pytest.skip("tests/dropin/_bin/ref_algorithms not built (the reference sources were absent at build time)")
    gf = tmp_path / "graph.bin"
    with open(gf, "wb") as f:
        np.array([g.n, g.nnz], np.int64).tofile(f)
        np.asarray(g.row_ptr, np.int32).tofile(f)
        np.asarray(g.col, np.int32).tofile(f)
        np.asarray(w, np.int32).tofile(f)
    out = tmp_path / "out"
    out.mkdir()
    log = tmp_path / "stdout.txt"
    with open(log, "w") as lf:
        res = subprocess.run([str(BIN), str(gf), str(out), str(int(source)), str(pr_iters)], stdout=lf,
                             stderr=subprocess.PIPE, text=True, cwd=tmp_path, timeout=600)
    text = log.read_text()
    assert res.returncode == 0, (res.stderr[-2000:], text[-2000:])
    assert "RESULTS" in text
    r = {}
    dt = {"bfs_blast": np.float32, "bfs_traditional": np.float32, "bfs_vanilla": np.int32, "cc": np.int32,
          "cc_bfs_based_sequential": np.int32, "pr": np.float32, "seq_page_rank": np.float32,
          "sssp_blast": np.float32, "sssp_gbkun": np.float32, "sssp_dijkstra": np.float32, "tc": np.uint64}
    for name, t in dt.items():
        r[name] = np.fromfile(out / f"{name}.bin", dtype=t)
    r["log"] = text
    return r


def seq_page_rank(g, iters, d=0.85):
    """pr_traditional.hpp:11-112 restated in FP64: in-degrees without self
    loops, the dangling mass of vertices without them spread evenly."""
    n = g.n
    rows = np.repeat(np.arange(n), np.diff(g.row_ptr))
    cols = np.asarray(g.col, np.int64)
    indeg = np.bincount(cols, minlength=n) - np.bincount(rows[rows == cols], minlength=n)
    inv = np.where(indeg > 0, 1.0 / np.maximum(indeg, 1), 0.0)
    keep = rows != cols
    r = np.full(n, 1.0 / n)
    for _ in range(iters):
        dangling = r[indeg <= 0].sum() / n
        acc = np.bincount(rows[keep], weights=(r * inv)[cols[keep]], minlength=n)
        r = (1.0 - d) / n + d * (acc + dangling)
    return r


def same_partition(a, b):
    """Two labelings describe the same components (a bijection of labels)."""
    pairs = set(zip(a.tolist(), b.tolist()))
    return len(pairs) == len(set(a.tolist())) == len(set(b.tolist()))


@pytest.mark.parametrize("name", ["rmat11u", "er11u"])
def test_reference_algorithms_match_reference_outputs(tmp_path, golden, name):
    data, _ = golden
    g = golden_graph(data, name)
    w = data[f"{name}.w"]
    src = int(data[f"{name}.sources"][0])
    r = run(tmp_path, g, w, src, 20)
    want_bfs = data[f"{name}.bfs.0"]
    assert np.array_equal(r["bfs_blast"], want_bfs.astype(np.float32))
    assert np.array_equal(r["bfs_traditional"], want_bfs.astype(np.float32))
    assert np.array_equal(r["bfs_vanilla"], want_bfs.astype(np.int32))
    assert np.array_equal(r["cc"], data[f"{name}.cc"])
    assert same_partition(r["cc_bfs_based_sequential"], data[f"{name}.cc"])
    assert rel_l1(r["pr"], data[f"{name}.pr.20"]) < REL_L1_TOL
    # the reference's sequential PageRank (pr_traditional.hpp:11-112) ran on the host CSR view
    assert rel_l1(r["seq_page_rank"], seq_page_rank(g, 20)) < REL_L1_TOL
    want_sssp = data[f"{name}.sssp"]
    assert np.array_equal(r["sssp_blast"], want_sssp)
    assert np.array_equal(r["sssp_gbkun"], want_sssp)
    assert np.array_equal(r["sssp_dijkstra"], want_sssp)
    tc = int(data[f"{name}.tc"][0])
    assert int(r["tc"][0]) == tc and int(r["tc"][1]) == tc
    assert int(r["tc"][2]) == 1 and "generic callable" in r["log"]
    assert "bfs_blast equals bfs_traditional: 1" in r["log"]


def test_reference_algorithms_rmat15_vs_oracle(tmp_path, oracle):
    g = gg.rmat(15, 16, seed=61, undirected=True)
    w = gg.weights_i32(g, seed=62)
    src = int(gg.sources(g, 1, seed=63)[0])
    r = run(tmp_path, g, w, src, 10)
    lv = oracle.bfs(g, src)
    assert np.array_equal(r["bfs_blast"], lv.astype(np.float32))
    assert np.array_equal(r["bfs_vanilla"], lv)
    assert np.array_equal(r["cc"], oracle.cc(g))
    d = oracle.sssp(g, w, src)
    want = np.where(d < 0, np.finfo(np.float32).max, d).astype(np.float32)
    assert np.array_equal(r["sssp_blast"], want)
    assert np.array_equal(r["sssp_dijkstra"], want)
    r64, _, _ = oracle.pagerank(g, tol=0.0, itermax=10)
    assert rel_l1(r["pr"], r64) < REL_L1_TOL
    assert int(r["tc"][0]) == oracle.tc(g)
    # the SAVE_STATS line of LAGraph_page_rank_sinks (pr.hpp:120) lands in perf_stats.txt
    stats = (tmp_path / "perf_stats.txt").read_text().splitlines()
    assert any(s.startswith("pr_mxv ") and "(GB/s)" in s for s in stats)
