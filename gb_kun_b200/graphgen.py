"""Seeded graph inputs: ctypes front end of ``libgbk_graphgen.so``.

The generator replaces the reference's time-seeded RMAT / random-uniform
generators (src/helpers/graph_generation/graph_generation.hpp:37-191) with a
counter-based one, so every run and every machine sees the same CSR.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_LIB = None


class _GbkGraph(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("row_ptr", C.POINTER(C.c_int32)),
                ("col", C.POINTER(C.c_int32))]


def _lib():
    global _LIB
    if _LIB is None:
        path = Path(__file__).resolve().parent / "libgbk_graphgen.so"
        if not path.exists():
            from . import build
            build.build_graphgen()
        lib = C.CDLL(str(path))
        gp = C.POINTER(C.POINTER(_GbkGraph))
        lib.gbk_gen_rmat.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int, gp]
        lib.gbk_gen_uniform.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_int, gp]
        lib.gbk_gen_from_edges.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, gp]
        lib.gbk_graph_free.argtypes = [C.POINTER(_GbkGraph)]
        lib.gbk_gen_values_f32.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        lib.gbk_gen_weights_i32.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_int32,
                                            C.c_void_p]
        lib.gbk_gen_vector_f32.argtypes = [C.c_int64, C.c_uint64, C.c_void_p]
        lib.gbk_gen_sources.argtypes = [C.c_int64, C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p]
        lib.gbk_gen_sources.restype = C.c_int64
        lib.gbk_gen_write_mtx.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                          C.c_void_p]
        lib.gbk_gen_write_mtxbin.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        _LIB = lib
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class Graph:
    """CSR graph: int32 row pointers and column ids (ascending within a row)."""
    n: int
    row_ptr: np.ndarray
    col: np.ndarray
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_ptr)


def _take(h) -> Graph:
    g = h.contents
    n, nnz = int(g.n), int(g.nnz)
    rp = np.ctypeslib.as_array(g.row_ptr, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(g.col, shape=(max(nnz, 1),))[:nnz].copy()
    _lib().gbk_graph_free(h)
    return Graph(n=n, row_ptr=rp, col=col)


def rmat(scale: int, edge_factor: int = 16, seed: int = 42, undirected: bool = False,
         a: float = 0.57, b: float = 0.19, c: float = 0.19) -> Graph:
    h = C.POINTER(_GbkGraph)()
    rc = _lib().gbk_gen_rmat(scale, edge_factor, a, b, c, seed, int(undirected), C.byref(h))
    if rc:
        raise RuntimeError(f"gbk_gen_rmat failed: {rc}")
    g = _take(h)
    g.name = f"rmat{scale}_ef{edge_factor}{'_u' if undirected else ''}_s{seed}"
    return g


def uniform(scale: int, edge_factor: int = 16, seed: int = 42, undirected: bool = False) -> Graph:
    h = C.POINTER(_GbkGraph)()
    rc = _lib().gbk_gen_uniform(scale, edge_factor, seed, int(undirected), C.byref(h))
    if rc:
        raise RuntimeError(f"gbk_gen_uniform failed: {rc}")
    g = _take(h)
    g.name = f"er{scale}_ef{edge_factor}{'_u' if undirected else ''}_s{seed}"
    return g


def from_edges(n: int, src, dst, undirected: bool = False) -> Graph:
    s = np.ascontiguousarray(src, dtype=np.int64)
    d = np.ascontiguousarray(dst, dtype=np.int64)
    h = C.POINTER(_GbkGraph)()
    rc = _lib().gbk_gen_from_edges(n, len(s), _p(s), _p(d), int(undirected), C.byref(h))
    if rc:
        raise RuntimeError(f"gbk_gen_from_edges failed: {rc}")
    return _take(h)


def values_f32(g: Graph, seed: int = 43) -> np.ndarray:
    out = np.empty(g.nnz, dtype=np.float32)
    _lib().gbk_gen_values_f32(g.n, _p(g.row_ptr), _p(g.col), seed, _p(out))
    return out


def weights_i32(g: Graph, seed: int = 43, lo: int = 1, hi: int = 255) -> np.ndarray:
    out = np.empty(g.nnz, dtype=np.int32)
    _lib().gbk_gen_weights_i32(g.n, _p(g.row_ptr), _p(g.col), seed, lo, hi, _p(out))
    return out


def vector_f32(n: int, seed: int = 44) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    _lib().gbk_gen_vector_f32(n, seed, _p(out))
    return out


def sources(g: Graph, count: int, seed: int = 45) -> np.ndarray:
    out = np.empty(count, dtype=np.int32)
    got = _lib().gbk_gen_sources(g.n, _p(g.row_ptr), count, seed, _p(out))
    return out[:got]


def edge_list(g: Graph):
    """(src, dst) int32 arrays of the CSR in row order."""
    return np.repeat(np.arange(g.n, dtype=np.int32), g.degrees()), np.ascontiguousarray(g.col, dtype=np.int32)


def write_mtx(path, nrows: int, ncols: int, src, dst, vals=None):
    """Matrix Market coordinate file of the edge list in the given order (1-based; a value column when
    vals is given)."""
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.ascontiguousarray(dst, dtype=np.int32)
    v = None if vals is None else np.ascontiguousarray(vals, dtype=np.float32)
    rc = _lib().gbk_gen_write_mtx(str(path).encode(), nrows, ncols, len(s), _p(s), _p(d),
                                  None if v is None else _p(v))
    if rc:
        raise RuntimeError(f"gbk_gen_write_mtx failed: {rc}")


def write_mtxbin(path, nrows: int, ncols: int, src, dst):
    """The reference's binary edge list: int64 rows, cols, nnz, then int64 1-based pairs."""
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.ascontiguousarray(dst, dtype=np.int32)
    rc = _lib().gbk_gen_write_mtxbin(str(path).encode(), nrows, ncols, len(s), _p(s), _p(d))
    if rc:
        raise RuntimeError(f"gbk_gen_write_mtxbin failed: {rc}")
