"""Host-side helpers of the query server (gb_kun_b200/serve.py) on the CPU:
the seeded Poisson request trace and the latency summary."""
import numpy as np

from gb_kun_b200.serve import KIND, QueryResult, latency_stats, poisson_trace


def test_poisson_trace_shape_rate_and_mix():
    cand = np.array([3, 5, 11, 17, 19], dtype=np.int32)
    arr, kinds, src = poisson_trace(20000, 500.0, mix=(0.5, 0.25, 0.25), candidates=cand, seed=3)
    assert arr.dtype == np.float64 and kinds.dtype == np.int32 and src.dtype == np.int32
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    # mean gap 1 / rate (2 ms) within a few percent over 20,000 requests
    assert abs(np.diff(arr).mean() - 2e-3) < 0.05 * 2e-3
    share = {k: float(np.mean(kinds == v)) for k, v in KIND.items()}
    assert abs(share["bfs"] - 0.5) < 0.02 and abs(share["sssp"] - 0.25) < 0.02 and abs(share["ppr"] - 0.25) < 0.02
    assert set(np.unique(src)) <= set(cand.tolist())


def test_poisson_trace_is_seeded_and_bounded():
    a = poisson_trace(100, 1000.0, n=50, seed=9)
    b = poisson_trace(100, 1000.0, n=50, seed=9)
    c = poisson_trace(100, 1000.0, n=50, seed=10)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.array_equal(a[2], c[2])
    assert a[2].min() >= 0 and a[2].max() < 50
    only_bfs = poisson_trace(50, 100.0, mix=(1.0, 0.0, 0.0), n=10, seed=1)[1]
    assert np.all(only_bfs == KIND["bfs"])
    empty = poisson_trace(0, 100.0, n=10)
    assert all(len(x) == 0 for x in empty)


def test_latency_stats_from_query_results():
    # the same structured array Server.run_trace returns
    res = np.ctypeslib.as_array((QueryResult * 101)()).copy()
    res["t_arrive"] = np.arange(101) * 0.01
    res["t_done"] = res["t_arrive"] + np.arange(101) * 1e-3  # latency i ms for request i
    st = latency_stats(res)
    for key, want in (("p50_ms", 50.0), ("p99_ms", 99.0), ("mean_ms", 50.0), ("max_ms", 100.0)):
        assert abs(st[key] - want) < 1e-9, key
