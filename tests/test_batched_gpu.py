"""GPU parity of the batched traversals (gbk_msbfs, gbk_ppr, gbk_sssp_multi).

Each lane must equal the single-source oracle for its source: BFS levels and
SSSP distances bit-exact, PPR within REL_L1_TOL of the FP64 oracle.  A lane's
result must not depend on the other lanes: one source alone and the same
source among others give identical output.
"""
import numpy as np
import pytest

from conftest import REL_L1_TOL, golden_graph, rel_l1
from gb_kun_b200 import graphgen as gg

pytestmark = pytest.mark.gpu

INF32 = np.iinfo(np.int32).max


@pytest.fixture(scope="module")
def torch():
    import torch as t
    from gb_kun_b200 import capi
    capi.init(0)
    return t


def _graphs():
    return [
        ("rmat12u", gg.rmat(12, 16, seed=5, undirected=True)),
        ("er12u", gg.uniform(12, 8, seed=6, undirected=True)),
        ("rmat11d", gg.rmat(11, 16, seed=7)),
        # isolated vertices, a path and a star hub (rows > 32 and > 256 entries)
        ("mixed", gg.from_edges(
            2000,
            np.concatenate([np.arange(0, 300), np.full(600, 500), np.arange(700, 1000)]),
            np.concatenate([np.arange(1, 301), np.arange(1000, 1600), np.arange(701, 1001)]),
            undirected=True)),
    ]


GRAPHS = _graphs()


def _mat(g, val=None):
    from gb_kun_b200 import capi
    return capi.Matrix.from_graph(g, val=val)


def _sources(g, k, seed):
    s = gg.sources(g, k, seed=seed)
    if len(s) < k:  # graphs with few non-isolated vertices: repeat
        s = np.resize(s, k)
    return s.astype(np.int32)


@pytest.mark.parametrize("name,g", GRAPHS, ids=[n for n, _ in GRAPHS])
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_msbfs_64_vs_oracle(torch, oracle, name, g, direction):
    A = _mat(g)
    src = _sources(g, 64, seed=21)
    src[5] = src[4]  # a duplicated source
    lv = torch.zeros((64, g.n), dtype=torch.int32, device="cuda")
    depths = A.msbfs(src, lv, direction=direction)
    got = lv.cpu().numpy()
    for k, s in enumerate(src):
        want = oracle.bfs(g, int(s))
        assert np.array_equal(got[k], want), (name, k, int(s))
        assert depths[k] == want.max()


def test_msbfs_few_sources_and_reuse(torch, oracle):
    _, g = GRAPHS[0]
    A = _mat(g)
    for k, seed in [(1, 30), (7, 31), (64, 32), (3, 33)]:
        src = _sources(g, k, seed=seed)
        lv = torch.full((k, g.n), -7, dtype=torch.int32, device="cuda")
        A.msbfs(src, lv)
        got = lv.cpu().numpy()
        for j, s in enumerate(src):
            assert np.array_equal(got[j], oracle.bfs(g, int(s)))


def test_msbfs_lane_independent(torch):
    _, g = GRAPHS[2]
    A = _mat(g)
    src = _sources(g, 64, seed=40)
    lv = torch.zeros((64, g.n), dtype=torch.int32, device="cuda")
    A.msbfs(src, lv)
    one = torch.zeros((1, g.n), dtype=torch.int32, device="cuda")
    A.msbfs(src[17:18], one)
    assert torch.equal(one[0], lv[17])


def test_msbfs_golden_reference(torch, golden):
    data, _ = golden
    for name in ["rmat11u", "er11u", "rmat10"]:
        g = golden_graph(data, name)
        A = _mat(g)
        src = np.asarray(data[f"{name}.sources"], dtype=np.int32)
        lv = torch.zeros((len(src), g.n), dtype=torch.int32, device="cuda")
        A.msbfs(src, lv)
        got = lv.cpu().numpy()
        for k in range(len(src)):
            assert np.array_equal(got[k], data[f"{name}.bfs.{k}"]), (name, k)


@pytest.mark.parametrize("name,g", GRAPHS, ids=[n for n, _ in GRAPHS])
def test_ppr_32_vs_oracle(torch, oracle, name, g):
    A = _mat(g)
    src = _sources(g, 32, seed=22)
    r = torch.zeros((32, g.n), dtype=torch.float32, device="cuda")
    # The iteration counts may differ from FP64 where FP32 rounding moves
    # sum |r_new - r| across tol (slowly converging paths); the ranks may not.
    A.ppr(src, r, damping=0.85, tol=1e-6, itermax=100)
    got = r.cpu().numpy()
    for k, s in enumerate(src):
        want, _ = oracle.ppr(g, int(s), damping=0.85, tol=1e-6, itermax=100)
        assert rel_l1(got[k], want) < REL_L1_TOL, (name, k, rel_l1(got[k], want))


def test_ppr_fixed_iterations_and_lane_independence(torch, oracle):
    _, g = GRAPHS[0]
    A = _mat(g)
    src = _sources(g, 32, seed=23)
    r = torch.zeros((32, g.n), dtype=torch.float32, device="cuda")
    iters = A.ppr(src, r, tol=0.0, itermax=7)
    assert (iters == 7).all()
    got = r.cpu().numpy()
    for k in (0, 13, 31):
        want, it = oracle.ppr(g, int(src[k]), tol=0.0, itermax=7)
        assert it == 7
        assert rel_l1(got[k], want) < REL_L1_TOL
    one = torch.zeros((1, g.n), dtype=torch.float32, device="cuda")
    A.ppr(src[13:14], one, tol=0.0, itermax=7)
    assert torch.equal(one[0], r[13])


@pytest.mark.parametrize("name,g", GRAPHS, ids=[n for n, _ in GRAPHS])
@pytest.mark.parametrize("vt", ["i32", "f32"])
def test_sssp_32_vs_oracle(torch, oracle, name, g, vt):
    w = gg.weights_i32(g, seed=3)
    A = _mat(g, val=w if vt == "i32" else w.astype(np.float32))
    src = _sources(g, 32, seed=24)
    d = torch.zeros((32, g.n), dtype=torch.int32, device="cuda")
    A.sssp_multi(src, d)
    got = d.cpu().numpy()
    for k, s in enumerate(src):
        want = oracle.sssp(g, w, int(s))
        assert np.array_equal(got[k], np.where(want < 0, INF32, want).astype(np.int32)), (name, k)


def test_sssp_lane_independent(torch):
    _, g = GRAPHS[0]
    w = gg.weights_i32(g, seed=4)
    A = _mat(g, val=w)
    src = _sources(g, 32, seed=25)
    d = torch.zeros((32, g.n), dtype=torch.int32, device="cuda")
    A.sssp_multi(src, d)
    one = torch.zeros((1, g.n), dtype=torch.int32, device="cuda")
    A.sssp_multi(src[9:10], one)
    assert torch.equal(one[0], d[9])


def test_batched_rejects_bad_input(torch):
    from gb_kun_b200 import capi
    _, g = GRAPHS[0]
    A = _mat(g)
    lv = torch.zeros((2, g.n), dtype=torch.int32, device="cuda")
    with pytest.raises(capi.GbkError) as e:
        A.msbfs(np.array([0, g.n], dtype=np.int32), lv)
    assert e.value.status == 6
    r = torch.zeros((33, g.n), dtype=torch.float32, device="cuda")
    with pytest.raises(capi.GbkError) as e:
        A.ppr(np.zeros(33, dtype=np.int32), r)
    assert e.value.status == 5
    # the matrix still works after the rejected calls
    A.msbfs(np.array([1], dtype=np.int32), lv[:1])


def test_batch_autotune_keeps_results(torch, oracle):
    _, g = GRAPHS[0]
    A = _mat(g, val=gg.weights_i32(g, seed=3))
    src = _sources(g, 64, seed=50)
    rb = A.batch_autotune("bfs", src)
    assert rb.ncandidates == 6 and rb.bfs_direction in (0, 1, 2) and rb.best_ms > 0
    rp = A.batch_autotune("ppr", src[:32])
    rs = A.batch_autotune("sssp", src[:32])
    assert rp.item_edges in (64, 128, 256, 512, 1024) and rs.item_edges in (64, 128, 256, 512, 1024)
    lv = torch.zeros((64, g.n), dtype=torch.int32, device="cuda")
    A.msbfs(src, lv)
    got = lv.cpu().numpy()
    for k in (0, 40):
        assert np.array_equal(got[k], oracle.bfs(g, int(src[k])))
    r = torch.zeros((32, g.n), dtype=torch.float32, device="cuda")
    A.ppr(src[:32], r)
    want, _ = oracle.ppr(g, int(src[3]), tol=1e-6, itermax=100)
    assert rel_l1(r[3].cpu().numpy(), want) < REL_L1_TOL


_HOST_LOOP_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from gb_kun_b200 import capi, graphgen as gg
capi.init(0)
g = gg.rmat(11, 16, seed=7)
A = capi.Matrix.from_graph(g, val=gg.weights_i32(g, seed=3))
src = gg.sources(g, 32, seed=60).astype(np.int32)
lv = torch.zeros((32, g.n), dtype=torch.int32, device="cuda"); A.msbfs(src, lv)
r = torch.zeros((32, g.n), dtype=torch.float32, device="cuda"); A.ppr(src, r)
d = torch.zeros((32, g.n), dtype=torch.int32, device="cuda"); A.sssp_multi(src, d)
np.savez(sys.argv[2], lv=lv.cpu().numpy(), r=r.cpu().numpy(), d=d.cpu().numpy())
"""


def test_host_loop_mode_matches_graph_mode(torch, tmp_path):
    """GBK_BATCH_HOST_LOOP=1 (for profilers) runs the same iteration kernels from the host."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    outs = {}
    for mode in ("0", "1"):
        f = tmp_path / f"m{mode}.npz"
        env = dict(os.environ, GBK_BATCH_HOST_LOOP=mode)
        res = subprocess.run([sys.executable, "-c", _HOST_LOOP_SCRIPT, str(root), str(f)], env=env,
                             capture_output=True, text=True, timeout=300)
        assert res.returncode == 0, res.stderr[-2000:]
        outs[mode] = np.load(f)
    for k in ("lv", "r", "d"):
        assert np.array_equal(outs["0"][k], outs["1"][k]), k
