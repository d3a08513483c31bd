"""ctypes binding of the query server (include/gbk_serve.h) and the request
trace used to drive it: Poisson arrivals of mixed BFS / SSSP / PPR queries
from uniformly drawn sources."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

KIND = {"bfs": 0, "ppr": 1, "sssp": 2}


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget", C.c_int64), ("max_batches", C.c_int32 * 3), ("lanes_per_batch", C.c_int32),
                ("max_inflight", C.c_int32), ("iters_per_launch", C.c_int32), ("keep_results", C.c_int32),
                ("ppr_damping", C.c_double), ("ppr_tol", C.c_double), ("ppr_itermax", C.c_int32)]


class QueryResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("kind", C.c_int32), ("source", C.c_int32), ("reached", C.c_int64),
                ("isum", C.c_int64), ("fsum", C.c_double), ("iters", C.c_int32), ("batch", C.c_int32),
                ("t_arrive", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


_DECLARED = False


def _lib():
    global _DECLARED
    L = capi.lib()
    if not _DECLARED:
        vp, i64 = C.c_void_p, C.c_int64
        L.gbk_server_create.argtypes = [vp, C.POINTER(ServerConfig), C.POINTER(vp)]
        L.gbk_server_destroy.argtypes = [vp]
        L.gbk_server_run_trace.argtypes = [vp, vp, vp, vp, i64, C.POINTER(QueryResult), C.POINTER(C.c_double)]
        L.gbk_server_fetch.argtypes = [vp, i64, vp]
        L.gbk_server_release.argtypes = [vp, i64]
        L.gbk_server_memory.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_int32)]
        for f in ("gbk_server_create", "gbk_server_destroy", "gbk_server_run_trace", "gbk_server_fetch",
                  "gbk_server_release", "gbk_server_memory"):
            getattr(L, f).restype = C.c_int
        _DECLARED = True
    return L


def poisson_trace(nq: int, rate_qps: float, mix=(0.5, 0.25, 0.25), candidates=None, n=None, seed=7):
    """Arrival times (s), kinds and sources of `nq` requests: exponential gaps of
    mean 1/rate_qps, kinds drawn with probabilities mix = (BFS, SSSP, PPR),
    sources uniform over `candidates` (e.g. non-isolated vertices) or [0, n)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_qps, size=nq))
    arrivals -= arrivals[0] if nq else 0.0
    p_bfs, p_sssp, p_ppr = mix
    kinds = rng.choice([KIND["bfs"], KIND["sssp"], KIND["ppr"]], size=nq, p=[p_bfs, p_sssp, p_ppr])
    if candidates is not None:
        sources = np.asarray(candidates)[rng.integers(0, len(candidates), size=nq)]
    else:
        sources = rng.integers(0, n, size=nq)
    return arrivals.astype(np.float64), kinds.astype(np.int32), sources.astype(np.int32)


class Server:
    """A query server over a resident capi.Matrix (values = integer SSSP weights)."""

    def __init__(self, A: capi.Matrix, memory_budget=0, max_batches=(1, 1, 1), lanes_per_batch=0,
                 max_inflight=0, iters_per_launch=4, keep_results=False, ppr_damping=0.85, ppr_tol=1e-6,
                 ppr_itermax=100):
        self.A = A
        cfg = ServerConfig(int(memory_budget), (C.c_int32 * 3)(*max_batches), int(lanes_per_batch),
                           int(max_inflight), int(iters_per_launch), int(bool(keep_results)), float(ppr_damping),
                           float(ppr_tol), int(ppr_itermax))
        self.h = C.c_void_p()
        capi.check(_lib().gbk_server_create(A.h, C.byref(cfg), C.byref(self.h)), "gbk_server_create")

    def close(self):
        if self.h:
            _lib().gbk_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_trace(self, arrivals, kinds, sources):
        """Replays the trace in real time; returns (structured results, wall seconds)."""
        arrivals = np.ascontiguousarray(arrivals, dtype=np.float64)
        kinds = np.ascontiguousarray(kinds, dtype=np.int32)
        sources = np.ascontiguousarray(sources, dtype=np.int32)
        nq = len(arrivals)
        out = (QueryResult * max(nq, 1))()
        wall = C.c_double(0)
        capi.check(_lib().gbk_server_run_trace(self.h, capi.ptr(kinds), capi.ptr(sources), capi.ptr(arrivals), nq,
                                               out, C.byref(wall)), "gbk_server_run_trace")
        res = np.ctypeslib.as_array(out)[:nq].copy()
        return res, wall.value

    def fetch(self, qid: int, kind: int) -> np.ndarray:
        dt = np.float32 if kind == KIND["ppr"] else np.int32
        dst = np.empty(self.A.n, dtype=dt)
        capi.check(_lib().gbk_server_fetch(self.h, int(qid), capi.ptr(dst)), "gbk_server_fetch")
        return dst

    def release(self, qid: int):
        capi.check(_lib().gbk_server_release(self.h, int(qid)), "gbk_server_release")

    def memory(self):
        used, budget, nb = C.c_int64(), C.c_int64(), C.c_int32()
        capi.check(_lib().gbk_server_memory(self.h, C.byref(used), C.byref(budget), C.byref(nb)),
                   "gbk_server_memory")
        return used.value, budget.value, nb.value


def latency_stats(res) -> dict:
    lat = (res["t_done"] - res["t_arrive"]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
