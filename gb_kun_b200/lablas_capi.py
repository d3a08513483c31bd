"""ctypes binding of libgbk_lablas.so: the reference's graph algorithms
(BFS, CC, SSSP, PageRank, triangle counting, SpMV) written against the
lablas:: C++ API and run on the GPU."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libgbk_lablas.so"
_LIB = None


class LablasError(RuntimeError):
    pass


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise LablasError(f"{LIB_PATH} is missing: run `python -m gb_kun_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        vp, i64, i32, dp = C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_double)
        L.gbk_lablas_graph_create.argtypes = [C.POINTER(vp), i64, vp, vp, vp]
        L.gbk_lablas_graph_destroy.argtypes = [vp]
        L.gbk_lablas_graph_from_file.argtypes = [C.POINTER(vp), C.c_char_p]
        L.gbk_lablas_get_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.gbk_lablas_bfs.argtypes = [vp, i64, vp, dp]
        L.gbk_lablas_cc.argtypes = [vp, vp, C.POINTER(i32), dp]
        L.gbk_lablas_bfs_ops.argtypes = [vp, i64, vp, dp]
        L.gbk_lablas_cc_fastsv.argtypes = [vp, vp, C.POINTER(i32), dp]
        L.gbk_lablas_sssp_f32.argtypes = [vp, i64, vp, dp]
        L.gbk_lablas_sssp_f32_ops.argtypes = [vp, i64, vp, dp]
        L.gbk_lablas_sssp_i32.argtypes = [vp, i64, vp, dp]
        L.gbk_lablas_pagerank.argtypes = [vp, i32, C.c_double, C.c_double, vp, C.POINTER(i32), dp]
        L.gbk_lablas_pagerank_ops.argtypes = [vp, i32, C.c_double, C.c_double, vp, C.POINTER(i32), dp]
        L.gbk_lablas_ppr.argtypes = [vp, i64, i32, C.c_double, C.c_double, vp, C.POINTER(i32), dp]
        L.gbk_lablas_tc.argtypes = [vp, C.POINTER(C.c_uint64), dp]
        L.gbk_lablas_tc_method.argtypes = [vp, i32, C.POINTER(C.c_uint64), dp]
        L.gbk_lablas_spmv.argtypes = [vp, i32, vp, vp, vp, dp]
        _LIB = L
    return _LIB


def _check(rc, where):
    if rc != 0:
        buf = C.create_string_buffer(1024)
        lib().gbk_lablas_get_last_error(buf, 1024)
        raise LablasError(f"{where}: status {rc}: {buf.value.decode(errors='replace')}")


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Graph:
    """A CSR graph resident on the device (lablas::Matrix<float> / <int>)."""

    def __init__(self, g, weights=None):
        from . import capi
        capi.init(0)
        self.n = g.n
        self._keep = (np.ascontiguousarray(g.row_ptr, np.int32), np.ascontiguousarray(g.col, np.int32),
                      None if weights is None else np.ascontiguousarray(weights, np.int32))
        self.h = C.c_void_p()
        rp, col, w = self._keep
        _check(lib().gbk_lablas_graph_create(C.byref(self.h), g.n, _p(rp), _p(col), _p(w)), "graph_create")

    @classmethod
    def from_file(cls, path) -> "Graph":
        """Graph from a .mtx / .mtxbin file or a .gbkcsr cache (lablas::Matrix<float>::init_from_mtx,
        parsed on the device; unit weights)."""
        from . import capi
        capi.init(0)
        self = cls.__new__(cls)
        self.n = int(capi.file_info(path).nrows)
        self._keep = None
        self.h = C.c_void_p()
        _check(lib().gbk_lablas_graph_from_file(C.byref(self.h), str(path).encode()), "graph_from_file")
        return self

    def close(self):
        if self.h:
            lib().gbk_lablas_graph_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bfs(self, source):
        out = np.empty(self.n, np.int32)
        ms = C.c_double()
        _check(lib().gbk_lablas_bfs(self.h, int(source), _p(out), C.byref(ms)), "bfs")
        return out, ms.value

    def bfs_ops(self, source):
        """bfs_blast as its sequence of GraphBLAS calls (one host read per level)."""
        out = np.empty(self.n, np.int32)
        ms = C.c_double()
        _check(lib().gbk_lablas_bfs_ops(self.h, int(source), _p(out), C.byref(ms)), "bfs_ops")
        return out, ms.value

    def cc(self):
        out = np.empty(self.n, np.int32)
        it = C.c_int32()
        ms = C.c_double()
        _check(lib().gbk_lablas_cc(self.h, _p(out), C.byref(it), C.byref(ms)), "cc")
        return out, ms.value

    def cc_fastsv(self):
        """The FastSV loop as the reference writes it; returns (labels, iterations, ms)."""
        out = np.empty(self.n, np.int32)
        it = C.c_int32()
        ms = C.c_double()
        _check(lib().gbk_lablas_cc_fastsv(self.h, _p(out), C.byref(it), C.byref(ms)), "cc_fastsv")
        return out, it.value, ms.value

    def sssp_f32(self, source):
        out = np.empty(self.n, np.float32)
        ms = C.c_double()
        _check(lib().gbk_lablas_sssp_f32(self.h, int(source), _p(out), C.byref(ms)), "sssp_f32")
        return out, ms.value

    def sssp_f32_ops(self, source):
        """sssp_bellman_ford_blast as its sequence of GraphBLAS calls (a host read per round)."""
        out = np.empty(self.n, np.float32)
        ms = C.c_double()
        _check(lib().gbk_lablas_sssp_f32_ops(self.h, int(source), _p(out), C.byref(ms)), "sssp_f32_ops")
        return out, ms.value

    def sssp_i32(self, source):
        out = np.empty(self.n, np.int32)
        ms = C.c_double()
        _check(lib().gbk_lablas_sssp_i32(self.h, int(source), _p(out), C.byref(ms)), "sssp_i32")
        return out, ms.value

    def pagerank(self, itermax=100, damping=0.85, tol=0.0):
        out = np.empty(self.n, np.float32)
        it = C.c_int32()
        ms = C.c_double()
        _check(lib().gbk_lablas_pagerank(self.h, itermax, damping, tol, _p(out), C.byref(it), C.byref(ms)),
               "pagerank")
        return out, it.value, ms.value

    def pagerank_ops(self, itermax=100, damping=0.85, tol=0.0):
        out = np.empty(self.n, np.float32)
        it = C.c_int32()
        ms = C.c_double()
        _check(lib().gbk_lablas_pagerank_ops(self.h, itermax, damping, tol, _p(out), C.byref(it), C.byref(ms)),
               "pagerank_ops")
        return out, it.value, ms.value

    def ppr(self, seed, itermax=100, damping=0.85, tol=1e-6):
        out = np.empty(self.n, np.float32)
        it = C.c_int32()
        ms = C.c_double()
        _check(lib().gbk_lablas_ppr(self.h, int(seed), itermax, damping, tol, _p(out), C.byref(it), C.byref(ms)),
               "ppr")
        return out, it.value, ms.value

    def tc(self):
        cnt = C.c_uint64()
        ms = C.c_double()
        _check(lib().gbk_lablas_tc(self.h, C.byref(cnt), C.byref(ms)), "tc")
        return int(cnt.value), ms.value

    def tc_method(self, method):
        """LAGr_TriangleCount with a method: 0 default, 1 Burkhardt, 2 Cohen, 3 Sandia, 4 Sandia2,
        5 SandiaDot, 6 SandiaDot2."""
        cnt = C.c_uint64()
        ms = C.c_double()
        _check(lib().gbk_lablas_tc_method(self.h, int(method), C.byref(cnt), C.byref(ms)), "tc_method")
        return int(cnt.value), ms.value

    def spmv(self, vals, x, fmt=0):
        y = np.empty(self.n, np.float32)
        ms = C.c_double()
        v = np.ascontiguousarray(vals, np.float32)
        xx = np.ascontiguousarray(x, np.float32)
        _check(lib().gbk_lablas_spmv(self.h, fmt, _p(v), _p(xx), _p(y), C.byref(ms)), "spmv")
        return y, ms.value


def bfs(g, source):
    return Graph(g).bfs(source)[0]
