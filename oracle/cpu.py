"""ctypes front end of the CPU checkers (TEST INFRASTRUCTURE ONLY).

* :class:`Oracle` wraps ``oracle/liboracle.so`` (the plain-C restatement).
* :class:`Reference` wraps ``oracle/_ref/libgbkref*.so`` (the reference's own
  CPU code compiled from its sources by ``oracle/Makefile``); it exists only
  where that build ran.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

SEMIRING = {"plus_times": 0, "lor_land": 1, "first_wins": 2, "first_min": 3, "plus_second": 4,
            "structural_bool": 5, "min_plus": 6, "custom_less_plus": 7, "min_second": 8, "min_noteq": 9,
            "plus_one": 10}
F32, I32 = 0, 1
MASK_DTYPE = {np.dtype(np.float32): 0, np.dtype(np.int32): 1, np.dtype(np.uint8): 2, np.dtype(np.bool_): 2,
              np.dtype(np.int64): 3, np.dtype(np.float64): 4}


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self):
        path = HERE / "liboracle.so"
        if not path.exists():
            import subprocess
            subprocess.run(["make", "-C", str(HERE), str(path)], check=True, capture_output=True)
        L = C.CDLL(str(path))
        vp, i64 = C.c_void_p, C.c_int64
        L.orc_spmv_f64.argtypes = [i64, vp, vp, vp, vp, vp]
        L.orc_mxv.argtypes = [C.c_int, C.c_int, C.c_int, i64, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int]
        L.orc_spmspv.argtypes = [C.c_int, C.c_int, C.c_int, i64, vp, vp, vp, i64, vp, vp, vp, vp, C.c_int,
                                 C.c_int]
        L.orc_bfs.argtypes = [i64, vp, vp, C.c_int32, vp]
        L.orc_cc.argtypes = [i64, vp, vp, vp]
        L.orc_sssp.argtypes = [i64, vp, vp, vp, C.c_int32, vp]
        L.orc_pagerank.argtypes = [i64, vp, vp, C.c_double, C.c_double, C.c_int, vp, vp]
        L.orc_pagerank.restype = C.c_int
        L.orc_ppr.argtypes = [i64, vp, vp, C.c_int32, C.c_double, C.c_double, C.c_int, vp]
        L.orc_ppr.restype = C.c_int
        L.orc_tc.argtypes = [i64, vp, vp]
        L.orc_tc.restype = C.c_uint64
        L.orc_transpose.argtypes = [i64, vp, vp, vp, vp, vp, vp]
        L.orc_read_graph_file.argtypes = [C.c_char_p, C.c_int, vp, vp, vp, vp, vp, vp]
        L.orc_read_graph_file.restype = C.c_int
        self.L = L

    def read_graph_file(self, path, kind=None):
        """(nrows, ncols, row_ptr, col) of a .mtx (kind 0) / .mtxbin (kind 1) file, rows in file order.
        Raises ValueError(code, bad_line) on a bad file."""
        if kind is None:
            kind = 1 if str(path).endswith("mtxbin") else 0
        r, c, z, bad = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_int64(0)
        rc = self.L.orc_read_graph_file(str(path).encode(), kind, C.byref(r), C.byref(c), C.byref(z), None, None,
                                        None)
        if rc:
            raise ValueError(rc, 0)
        rp = np.empty(r.value + 1, np.int32)
        col = np.empty(max(z.value, 1), np.int32)
        rc = self.L.orc_read_graph_file(str(path).encode(), kind, C.byref(r), C.byref(c), C.byref(z), _p(rp),
                                        _p(col), C.byref(bad))
        if rc:
            raise ValueError(rc, bad.value)
        return r.value, c.value, rp, col[:z.value]

    def spmv_f64(self, g, val, x):
        y = np.empty(g.n, dtype=np.float64)
        self.L.orc_spmv_f64(g.n, _p(g.row_ptr), _p(g.col), _p(val), _p(x), _p(y))
        return y

    def mxv(self, semiring, g, val, x, y_in, accum=0, mask=None, mask_mode=6):
        dt = F32 if val.dtype == np.float32 else I32
        y = y_in.copy()
        md = MASK_DTYPE[mask.dtype] if mask is not None else 0
        mk = mask.view(np.uint8) if (mask is not None and mask.dtype == np.bool_) else mask
        self.L.orc_mxv(SEMIRING[semiring] if isinstance(semiring, str) else semiring, accum, dt, g.n,
                       _p(g.row_ptr), _p(g.col), _p(val), _p(x), _p(y), _p(mk), md, mask_mode)
        return y

    def spmspv(self, semiring, g, val, f_ids, f_vals, y_in, accum=0, mask=None, mask_mode=6):
        dt = F32 if val.dtype == np.float32 else I32
        y = y_in.copy()
        md = MASK_DTYPE[mask.dtype] if mask is not None else 0
        mk = mask.view(np.uint8) if (mask is not None and mask.dtype == np.bool_) else mask
        self.L.orc_spmspv(SEMIRING[semiring] if isinstance(semiring, str) else semiring, accum, dt, g.n,
                          _p(g.row_ptr), _p(g.col), _p(val), len(f_ids), _p(f_ids), _p(f_vals), _p(y), _p(mk),
                          md, mask_mode)
        return y

    def bfs(self, g, source):
        lv = np.empty(g.n, dtype=np.int32)
        self.L.orc_bfs(g.n, _p(g.row_ptr), _p(g.col), int(source), _p(lv))
        return lv

    def cc(self, g):
        lab = np.empty(g.n, dtype=np.int32)
        self.L.orc_cc(g.n, _p(g.row_ptr), _p(g.col), _p(lab))
        return lab

    def sssp(self, g, w, source):
        d = np.empty(g.n, dtype=np.int64)
        self.L.orc_sssp(g.n, _p(g.row_ptr), _p(g.col), _p(w), int(source), _p(d))
        return d

    def pagerank(self, g, damping=0.85, tol=0.0, itermax=100):
        r = np.empty(g.n, dtype=np.float64)
        last = C.c_double(0)
        it = self.L.orc_pagerank(g.n, _p(g.row_ptr), _p(g.col), damping, tol, itermax, _p(r), C.byref(last))
        return r, it, last.value

    def ppr(self, g, seed, damping=0.85, tol=0.0, itermax=100):
        r = np.empty(g.n, dtype=np.float64)
        it = self.L.orc_ppr(g.n, _p(g.row_ptr), _p(g.col), int(seed), damping, tol, itermax, _p(r))
        return r, it

    def tc(self, g):
        return int(self.L.orc_tc(g.n, _p(g.row_ptr), _p(g.col)))

    def transpose(self, g, val=None):
        cp = np.empty(g.n + 1, dtype=np.int32)
        row = np.empty(max(g.nnz, 1), dtype=np.int32)
        tv = np.empty(max(g.nnz, 1), dtype=np.float32) if val is not None else None
        self.L.orc_transpose(g.n, _p(g.row_ptr), _p(g.col), _p(val), _p(cp), _p(row), _p(tv))
        return cp, row[:g.nnz], (tv[:g.nnz] if tv is not None else None)


class Reference:
    """The reference's own CPU implementation (built from its sources)."""

    def __init__(self):
        self.path = HERE / "_ref" / "libgbkref.so"
        self.path_cc = HERE / "_ref" / "libgbkref_cc.so"
        if not self.path.exists():
            raise FileNotFoundError(str(self.path))
        vp, i64, i32, dp = C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_double)
        self.L = C.CDLL(str(self.path))
        self.Lcc = C.CDLL(str(self.path_cc))
        for L in (self.L, self.Lcc):
            L.ref_spmv.argtypes = [C.c_int, C.c_int, i64, vp, vp, vp, vp, vp, C.c_int, C.c_int, dp]
            L.ref_bfs.argtypes = [i64, vp, vp, i32, vp, C.c_int, dp]
            L.ref_cc.argtypes = [i64, vp, vp, vp, C.c_int, dp]
            L.ref_sssp.argtypes = [i64, vp, vp, vp, i32, vp, C.c_int, dp]
            L.ref_pr.argtypes = [i64, vp, vp, C.c_int, vp, C.c_int, dp]
            L.ref_tc.argtypes = [i64, vp, vp, vp, C.c_int, dp]
            L.ref_max_threads.restype = C.c_int
            L.ref_graph_read.argtypes = [C.c_char_p, C.POINTER(i64), C.POINTER(i64), C.POINTER(vp), dp]
            L.ref_graph_csr.argtypes = [vp, vp, vp, vp]
            L.ref_graph_free.argtypes = [vp]
            L.ref_mxm.argtypes = [C.c_int, i64, vp, vp, vp, C.POINTER(vp), C.POINTER(i64), dp]
            L.ref_tc_method.argtypes = [C.c_int, i64, vp, vp, vp, dp]
            L.ref_select_matrix.argtypes = [C.c_int, C.c_double, i64, vp, vp, vp, C.POINTER(vp)]

    @staticmethod
    def available() -> bool:
        return (HERE / "_ref" / "libgbkref.so").exists() and (HERE / "_ref" / "libgbkref_cc.so").exists()

    def max_threads(self) -> int:
        return int(self.L.ref_max_threads())

    def spmv(self, g, val, x, fmt=0, semiring=0, warmup=0, reps=1):
        y = np.empty(g.n, dtype=np.float32)
        ms = C.c_double(0)
        rc = self.L.ref_spmv(fmt, semiring, g.n, _p(g.row_ptr), _p(g.col), _p(val), _p(x), _p(y), warmup, reps,
                             C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_spmv rc={rc}")
        return y, ms.value

    def bfs(self, g, source, reps=1):
        lv = np.empty(g.n, dtype=np.int32)
        ms = C.c_double(0)
        rc = self.L.ref_bfs(g.n, _p(g.row_ptr), _p(g.col), int(source), _p(lv), reps, C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_bfs rc={rc}")
        return lv, ms.value

    def cc(self, g, reps=1):
        lab = np.empty(g.n, dtype=np.int32)
        ms = C.c_double(0)
        rc = self.Lcc.ref_cc(g.n, _p(g.row_ptr), _p(g.col), _p(lab), reps, C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_cc rc={rc}")
        return lab, ms.value

    def sssp(self, g, w, source, reps=1):
        d = np.empty(g.n, dtype=np.float32)
        ms = C.c_double(0)
        rc = self.L.ref_sssp(g.n, _p(g.row_ptr), _p(g.col), _p(w), int(source), _p(d), reps, C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_sssp rc={rc}")
        return d, ms.value

    def pagerank(self, g, iters, reps=1):
        r = np.empty(g.n, dtype=np.float32)
        ms = C.c_double(0)
        rc = self.L.ref_pr(g.n, _p(g.row_ptr), _p(g.col), int(iters), _p(r), reps, C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_pr rc={rc}")
        return r, ms.value

    def tc(self, g, reps=1):
        cnt = C.c_uint64(0)
        ms = C.c_double(0)
        rc = self.L.ref_tc(g.n, _p(g.row_ptr), _p(g.col), C.byref(cnt), reps, C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_tc rc={rc}")
        return int(cnt.value), ms.value

    def graph_read(self, path):
        """The reference's Matrix<float>::init_from_mtx: (nrows, row_ptr, col, val, ms)."""
        n, z, h, ms = C.c_int64(0), C.c_int64(0), C.c_void_p(), C.c_double(0)
        rc = self.L.ref_graph_read(str(path).encode(), C.byref(n), C.byref(z), C.byref(h), C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_graph_read rc={rc}")
        try:
            rp = np.empty(n.value + 1, np.int32)
            col = np.empty(max(z.value, 1), np.int32)
            val = np.empty(max(z.value, 1), np.float32)
            self.L.ref_graph_csr(h, _p(rp), _p(col), _p(val))
        finally:
            self.L.ref_graph_free(h)
        return n.value, rp, col[:z.value], val[:z.value], ms.value

    def _take_matrix(self, h, n, nnz):
        """(row_ptr, col, val) of a reference matrix (n rows, nnz entries) behind handle h, freed afterwards."""
        try:
            rp = np.empty(n + 1, np.int32)
            col = np.empty(max(nnz, 1), np.int32)
            val = np.empty(max(nnz, 1), np.float32)
            self.L.ref_graph_csr(h, _p(rp), _p(col), _p(val))
        finally:
            self.L.ref_graph_free(h)
        return rp, col[:nnz], val[:nnz]

    def mxm(self, g, val, semiring=0):
        """The reference's unmasked A (+.x) A: (row_ptr, col, val, ms), rows in its hash-map order."""
        h, z, ms = C.c_void_p(), C.c_int64(0), C.c_double(0)
        rc = self.L.ref_mxm(semiring, g.n, _p(g.row_ptr), _p(g.col), _p(val), C.byref(h), C.byref(z), C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_mxm rc={rc}")
        rp, col, v = self._take_matrix(h, g.n, z.value)
        return rp, col, v, ms.value

    def select_matrix(self, g, val, op, thunk):
        h = C.c_void_p()
        rc = self.L.ref_select_matrix(op, float(thunk), g.n, _p(g.row_ptr), _p(g.col), _p(val), C.byref(h))
        if rc:
            raise RuntimeError(f"ref_select_matrix rc={rc}")
        return self._take_matrix(h, g.n, g.nnz)

    def tc_method(self, g, method):
        cnt, ms = C.c_uint64(0), C.c_double(0)
        rc = self.L.ref_tc_method(method, g.n, _p(g.row_ptr), _p(g.col), C.byref(cnt), C.byref(ms))
        if rc:
            raise RuntimeError(f"ref_tc_method rc={rc}")
        return int(cnt.value), ms.value
