"""ctypes binding of the gbk C ABI (libgbk.so) for Python callers.

Device vectors are passed as raw device pointers; :mod:`torch` tensors are the
convenient owner of that memory (``tensor.data_ptr()``) but never cross the
ABI.  Every non-zero status raises :class:`GbkError` with the library's last
error text.  There is no CPU fallback: if the CUDA library is missing or no
sm_100 device is present, calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libgbk.so"

# gbk_types.h
F32, I32, BOOL, I64, F64 = 0, 1, 2, 3, 4
FMT = {"CSR": 0, "CSR_SEG": 3, "LAV": 4, "SELL_C": 6}
SEMIRING = {"plus_times": 0, "lor_land": 1, "first_wins": 2, "first_min": 3, "plus_second": 4,
            "structural_bool": 5, "min_plus": 6, "custom_less_plus": 7, "min_second": 8, "min_noteq": 9,
            "plus_one": 10}
BINOP = {"second": 0, "first": 1, "plus": 2, "minus": 3, "times": 4, "div": 5, "min": 6, "max": 7, "lor": 8,
         "land": 9, "ne": 10, "lt": 11, "one": 12}
UNOP = {"identity": 0, "abs": 1, "one": 2}
MASK = {"scmp": 0, "comp": 2, "structure": 4, "str_comp": 5, "default": 6}
MONOID = {"plus": 0, "min": 1, "max": 2, "lor": 3, "land": 4, "times": 5}
SELECT = {"tril": 0, "triu": 1, "diag": 2, "offdiag": 3, "value_eq": 4, "value_ne": 5, "value_gt": 6,
          "value_ge": 7, "value_lt": 8, "value_le": 9}


class GbkError(RuntimeError):
    def __init__(self, status: int, where: str, text: str):
        super().__init__(f"{where}: status {status}: {text}")
        self.status = status


class BatchTuneResult(C.Structure):
    _fields_ = [("kind", C.c_int32), ("item_edges", C.c_int32), ("bfs_direction", C.c_int32),
                ("bfs_alpha", C.c_int32), ("ncandidates", C.c_int32), ("best_ms", C.c_float),
                ("candidate_ms", C.c_float * 8)]

    def describe(self) -> dict:
        return {"kind": ["bfs", "ppr", "sssp"][self.kind], "item_edges": self.item_edges,
                "bfs_direction": self.bfs_direction, "bfs_alpha": self.bfs_alpha, "best_ms": round(self.best_ms, 3),
                "candidate_ms": [round(x, 3) for x in list(self.candidate_ms)[:self.ncandidates]]}


class FormatParams(C.Structure):
    _fields_ = [("sell_c", C.c_int32), ("sell_sigma", C.c_int32), ("seg_cols", C.c_int32),
                ("lav_dense_frac", C.c_float), ("csr_kernel", C.c_int32), ("sell_hot_cols", C.c_int32),
                ("sell_reorder_cols", C.c_int32), ("seg_staged", C.c_int32)]


class MatrixInfo(C.Structure):
    _fields_ = [("nrows", C.c_int64), ("ncols", C.c_int64), ("nnz", C.c_int64), ("vtype", C.c_int32),
                ("format", C.c_int32), ("padded_nnz", C.c_int64), ("device_bytes", C.c_int64),
                ("ntiles", C.c_int64), ("has_csc", C.c_int32)]


class TuneResult(C.Structure):
    _fields_ = [("format", C.c_int32), ("sell_sigma", C.c_int32), ("csr_kernel", C.c_int32), ("cached", C.c_int32),
                ("ncandidates", C.c_int32), ("best_ms", C.c_float), ("candidate_ms", C.c_float * 16),
                ("sell_hot_cols", C.c_int32), ("sell_staged", C.c_int32)]

    CANDIDATES = ["CSR_bins", "CSR_merge", "SELL_C_s1", "SELL_C_s256", "SELL_C_s4096", "CSR_SEG", "LAV",
                  "SELL_C_s4096_hot16k", "SELL_C_s4096_hot52k", "SELL_C_s256_hot52k", "SELL_C_s4096_reorder",
                  "SELL_C_s256_reorder", "SELL_C_staged", "SELL_C_staged_reorder", "CSR_chunks"]

    def describe(self) -> dict:
        names = {0: "CSR", 3: "CSR_SEG", 4: "LAV", 6: "SELL_C"}
        d = {"format": names.get(self.format, str(self.format)), "cached": bool(self.cached)}
        if self.format == 6:
            d["sigma"] = self.sell_sigma
            d["hot_cols"] = self.sell_hot_cols
            d["staged_windows"] = bool(self.sell_staged)
        if self.format == 0:
            d["csr_kernel"] = {1: "merge-path", 2: "degree-bins", 3: "entry-chunks"}.get(self.csr_kernel, "default")
        if not self.cached:
            d["candidate_ms"] = {n: round(self.candidate_ms[i], 4) for i, n in enumerate(self.CANDIDATES)
                                 if i < self.ncandidates}
        return d


class FileInfo(C.Structure):
    _fields_ = [("nrows", C.c_int64), ("ncols", C.c_int64), ("nnz", C.c_int64), ("file_bytes", C.c_int64),
                ("data_offset", C.c_int64), ("kind", C.c_int32), ("vtype", C.c_int32)]

    KINDS = {0: "mtx", 1: "mtxbin", 2: "csr"}


class Mask(C.Structure):
    """gbk_mask: dense (dense != NULL) or sparse (ids, nvals) mask argument."""
    _fields_ = [("dense", C.c_void_p), ("dtype", C.c_int32), ("mode", C.c_int32), ("ids", C.c_void_p),
                ("nvals", C.c_int64)]


_LIB = None


def _declare(lib):
    vp, i64, i32, ci = C.c_void_p, C.c_int64, C.c_int32, C.c_int
    mp = C.POINTER(Mask)
    sig = {
        "gbk_mxv_sparse_mask": ([vp, ci, ci, ci, ci, vp, vp, vp, i64, ci, vp], ci),
        "gbk_spmspv": ([vp, ci, ci, ci, ci, vp, vp, i64, vp, mp, vp], ci),
        "gbk_spmspv_sparse": ([vp, ci, ci, ci, vp, vp, i64, vp, vp, C.POINTER(i64), mp, vp], ci),
        "gbk_mxm_masked": ([C.POINTER(vp), vp, vp, vp, ci, ci, vp], ci),
        "gbk_matrix_autotune": ([vp, ci, ci, i32, C.POINTER(TuneResult), vp], ci),
        "gbk_vec_nvals": ([vp, ci, i64, C.POINTER(i64), vp], ci),
        "gbk_vec_to_sparse": ([vp, ci, i64, vp, vp, C.POINTER(i64), vp], ci),
        "gbk_vec_to_dense": ([vp, vp, i64, ci, vp, i64, vp], ci),
        "gbk_vec_fill": ([vp, ci, i64, C.c_double, vp], ci),
        "gbk_vec_iota": ([vp, ci, i64, vp], ci),
        "gbk_vec_cast": ([vp, ci, vp, ci, i64, vp], ci),
        "gbk_ewise": ([ci, ci, vp, ci, vp, ci, vp, ci, i64, mp, vp], ci),
        "gbk_apply": ([ci, ci, ci, vp, ci, vp, ci, C.c_double, i64, mp, vp], ci),
        "gbk_assign_scalar": ([vp, ci, i64, C.c_double, mp, vp, ci, i64, vp], ci),
        "gbk_assign_vector": ([ci, ci, vp, ci, vp, ci, i64, mp, vp, ci, i64, vp], ci),
        "gbk_extract": ([ci, ci, vp, ci, vp, ci, i64, mp, vp, ci, i64, vp], ci),
        "gbk_reduce": ([ci, ci, vp, ci, i64, vp, vp], ci),
        "gbk_init": ([ci], ci),
        "gbk_get_last_error": ([C.c_char_p, C.c_size_t], ci),
        "gbk_launch_count": ([], i64),
        "gbk_matrix_create_csr": ([C.POINTER(vp), i64, i64, i64, vp, vp, vp, ci, ci, vp], ci),
        "gbk_matrix_destroy": ([vp], ci),
        "gbk_matrix_get_info": ([vp, C.POINTER(MatrixInfo)], ci),
        "gbk_matrix_csr_arrays": ([vp, ci, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), vp], ci),
        "gbk_matrix_set_format": ([vp, ci, C.POINTER(FormatParams), vp], ci),
        "gbk_mxv": ([vp, ci, ci, ci, ci, vp, vp, vp, ci, ci, vp], ci),
        "gbk_msbfs": ([vp, vp, ci, vp, ci, vp, vp], ci),
        "gbk_ppr": ([vp, vp, ci, C.c_double, C.c_double, ci, vp, vp, vp], ci),
        "gbk_sssp_multi": ([vp, vp, ci, vp, vp, vp], ci),
        "gbk_bfs_levels": ([vp, i64, ci, ci, vp, C.POINTER(i32), vp], ci),
        "gbk_matrix_pattern_symmetric": ([vp, C.POINTER(i32), vp], ci),
        "gbk_cc_labels": ([vp, ci, vp, vp], ci),
        "gbk_sssp_dist": ([vp, i64, C.c_double, vp, C.POINTER(i32), vp], ci),
        "gbk_pagerank": ([vp, i32, C.c_double, C.c_double, vp, C.POINTER(i32), C.POINTER(C.c_float), vp], ci),
        "gbk_batch_autotune": ([vp, ci, vp, ci, C.POINTER(BatchTuneResult), vp], ci),
        "gbk_mxm": ([C.POINTER(vp), vp, vp, ci, vp], ci),
        "gbk_triangle_count": ([vp, C.POINTER(C.c_uint64), vp], ci),
        "gbk_select_matrix": ([C.POINTER(vp), vp, ci, C.c_double, vp], ci),
        "gbk_select_vector": ([ci, C.c_double, vp, ci, vp, ci, i64, ci, mp, ci, vp], ci),
        "gbk_file_info_read": ([C.c_char_p, C.POINTER(FileInfo)], ci),
        "gbk_matrix_create_from_file": ([C.POINTER(vp), C.c_char_p, ci, vp], ci),
        "gbk_matrix_save_csr": ([vp, C.c_char_p, vp], ci),
        "gbk_matrix_load_csr": ([C.POINTER(vp), C.c_char_p, vp], ci),
        "gbk_matrix_download_csr": ([vp, vp, vp, vp, vp], ci),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res
    return lib


def lib():
    """Load libgbk.so (built in-tree by gb_kun_b200.build)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise GbkError(-1, "load", f"{LIB_PATH} is missing: run `python -m gb_kun_b200.build`")
        _LIB = _declare(C.CDLL(str(LIB_PATH)))
    return _LIB


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().gbk_get_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, where: str):
    if status != 0:
        raise GbkError(status, where, last_error())


def init(device: int = 0):
    check(lib().gbk_init(device), "gbk_init")


def select_vector(w, u, op: str, thunk=0.0, accum="second", mask=None, mask_mode="default", replace=False,
                  stream=None):
    """w[i] = accum(w[i], u[i] if op keeps (u[i], i) else 0) where the dense mask selects (all i without one)."""
    m = None
    if mask is not None:
        m = Mask(ptr(mask), dtype_code(mask), MASK[mask_mode], None, 0)
    check(lib().gbk_select_vector(SELECT[op], float(thunk), ptr(w), dtype_code(w), ptr(u), dtype_code(u),
                                  int(w.numel()), BINOP[accum], None if m is None else C.byref(m), int(replace),
                                  stream_ptr(stream)), "gbk_select_vector")
    return w


def file_info(path) -> FileInfo:
    """Header of a .mtx / .mtxbin / .gbkcsr file."""
    inf = FileInfo()
    check(lib().gbk_file_info_read(str(path).encode(), C.byref(inf)), "gbk_file_info_read")
    return inf


def launch_count() -> int:
    return int(lib().gbk_launch_count())


def ptr(t) -> C.c_void_p | None:
    """Device (or host) address of a torch tensor / numpy array, None for None."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return C.c_void_p(t.ctypes.data)
    return C.c_void_p(t.data_ptr())


def dtype_code(t) -> int:
    import torch
    m = {torch.float32: F32, torch.int32: I32, torch.bool: BOOL, torch.uint8: BOOL, torch.int64: I64,
         torch.float64: F64}
    return m[t.dtype]


def stream_ptr(stream=None):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Matrix:
    """Device matrix handle (CSR + lazily built CSC + optional format)."""

    def __init__(self, row_ptr: np.ndarray, col: np.ndarray, val: np.ndarray, ncols: int | None = None,
                 stream=None):
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val)
        vt = {np.dtype(np.float32): F32, np.dtype(np.int32): I32}[val.dtype]
        self.n = len(row_ptr) - 1
        self.ncols = self.n if ncols is None else ncols
        self.nnz = int(row_ptr[-1])
        self.vtype = vt
        self.h = C.c_void_p()
        check(lib().gbk_matrix_create_csr(C.byref(self.h), self.n, self.ncols, self.nnz, ptr(row_ptr), ptr(col),
                                          ptr(val), vt, 0, stream_ptr(stream)), "gbk_matrix_create_csr")

    @classmethod
    def from_graph(cls, g, val=None, stream=None):
        if val is None:
            val = np.ones(g.nnz, dtype=np.float32)
        return cls(g.row_ptr, g.col, val, stream=stream)

    @classmethod
    def _adopt(cls, h) -> "Matrix":
        m = cls.__new__(cls)
        m.h = h
        inf = m.info()
        m.n, m.ncols, m.nnz, m.vtype = int(inf.nrows), int(inf.ncols), int(inf.nnz), int(inf.vtype)
        return m

    @classmethod
    def from_file(cls, path, dtype="f32", stream=None) -> "Matrix":
        """Matrix from a .mtx / .mtxbin graph file (parsed on the device, every value 1) or a
        .gbkcsr CSR cache (Matrix<T>::init_from_mtx)."""
        h = C.c_void_p()
        check(lib().gbk_matrix_create_from_file(C.byref(h), str(path).encode(), {"f32": F32, "i32": I32}[dtype],
                                                stream_ptr(stream)), "gbk_matrix_create_from_file")
        return cls._adopt(h)

    @classmethod
    def load_csr(cls, path, stream=None) -> "Matrix":
        h = C.c_void_p()
        check(lib().gbk_matrix_load_csr(C.byref(h), str(path).encode(), stream_ptr(stream)), "gbk_matrix_load_csr")
        return cls._adopt(h)

    def save_csr(self, path, stream=None):
        check(lib().gbk_matrix_save_csr(self.h, str(path).encode(), stream_ptr(stream)), "gbk_matrix_save_csr")

    def mxm(self, B: "Matrix", semiring="plus_times", stream=None) -> "Matrix":
        """Unmasked C = self (+.x) B (SpMSpM_unmasked_ikj); zero sums dropped, rows column-sorted."""
        h = C.c_void_p()
        check(lib().gbk_mxm(C.byref(h), self.h, B.h, SEMIRING[semiring], stream_ptr(stream)), "gbk_mxm")
        return Matrix._adopt(h)

    def triangle_count(self, stream=None) -> int:
        """Burkhardt's sum((A*A) .* A) / 6 (oriented count on a symmetric loop-free A)."""
        c = C.c_uint64(0)
        check(lib().gbk_triangle_count(self.h, C.byref(c), stream_ptr(stream)), "gbk_triangle_count")
        return int(c.value)

    def select(self, op: str, thunk=0.0, stream=None) -> "Matrix":
        """Matrix select (select.h:363-395): same structure, values kept where op keeps them, else 0."""
        h = C.c_void_p()
        check(lib().gbk_select_matrix(C.byref(h), self.h, SELECT[op], float(thunk), stream_ptr(stream)),
              "gbk_select_matrix")
        return Matrix._adopt(h)

    def download_csr(self, stream=None):
        """(row_ptr, col, val) of the CSR as host numpy arrays."""
        rp = np.empty(self.n + 1, np.int32)
        col = np.empty(max(self.nnz, 1), np.int32)
        val = np.empty(max(self.nnz, 1), np.float32 if self.vtype == F32 else np.int32)
        check(lib().gbk_matrix_download_csr(self.h, ptr(rp), ptr(col), ptr(val), stream_ptr(stream)),
              "gbk_matrix_download_csr")
        return rp, col[:self.nnz], val[:self.nnz]

    def close(self):
        if self.h:
            lib().gbk_matrix_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> MatrixInfo:
        inf = MatrixInfo()
        check(lib().gbk_matrix_get_info(self.h, C.byref(inf)), "gbk_matrix_get_info")
        return inf

    def set_format(self, fmt: str, sell_c=0, sigma=0, seg_cols=0, lav_frac=0.0, csr_kernel=0, hot_cols=0,
                   reorder_cols=0, seg_staged=0, stream=None):
        """Storage format; csr_kernel picks the CSR kernel (0 default: bins, or runs of 256 entries
        for unmasked products over 2^23+ entries; 1 merge-path, 2 bins, 3 runs of 256 entries per warp);
        hot_cols > 0 stages the x values of the most used columns in shared memory (SELL-C);
        reorder_cols renumbers columns by in-degree (SELL-C)."""
        p = FormatParams(sell_c, sigma, seg_cols, lav_frac, csr_kernel, hot_cols, reorder_cols, seg_staged)
        check(lib().gbk_matrix_set_format(self.h, FMT[fmt], C.byref(p), stream_ptr(stream)), "gbk_matrix_set_format")

    def autotune(self, transpose=False, semiring="plus_times", reps=20, stream=None) -> TuneResult:
        """Time every format / kernel candidate and keep the fastest on this matrix."""
        r = TuneResult()
        check(lib().gbk_matrix_autotune(self.h, int(transpose), SEMIRING[semiring], reps, C.byref(r),
                                        stream_ptr(stream)), "gbk_matrix_autotune")
        return r

    def arrays(self, transpose=False, stream=None):
        p, i, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().gbk_matrix_csr_arrays(self.h, int(transpose), C.byref(p), C.byref(i), C.byref(v),
                                          stream_ptr(stream)), "gbk_matrix_csr_arrays")
        return p.value, i.value, v.value

    def mxv(self, x, y, semiring="plus_times", accum="second", mask=None, mask_mode="default", transpose=False,
            stream=None):
        """y = accum(y, A x) (transpose=False) or accum(y, A^T x) on device tensors."""
        check(lib().gbk_mxv(self.h, int(transpose), SEMIRING[semiring], BINOP[accum], dtype_code(y), ptr(x), ptr(y),
                            ptr(mask), dtype_code(mask) if mask is not None else 0, MASK[mask_mode],
                            stream_ptr(stream)), "gbk_mxv")
        return y

    def mxv_sparse_mask(self, x, y, mask_ids, semiring="plus_times", accum="second", mask_mode="default",
                        transpose=False, stream=None):
        check(lib().gbk_mxv_sparse_mask(self.h, int(transpose), SEMIRING[semiring], BINOP[accum], dtype_code(y),
                                        ptr(x), ptr(y), ptr(mask_ids), int(mask_ids.numel()), MASK[mask_mode],
                                        stream_ptr(stream)), "gbk_mxv_sparse_mask")
        return y

    def spmspv(self, x_ids, x_vals, y, semiring="lor_land", accum="second", mask=None, transpose=False,
               stream=None):
        """Push SpMSpV from the sparse vector (x_ids, x_vals) into dense y."""
        check(lib().gbk_spmspv(self.h, int(transpose), SEMIRING[semiring], BINOP[accum], dtype_code(y), ptr(x_ids),
                               ptr(x_vals), int(x_ids.numel()), ptr(y), C.byref(mask) if mask is not None else None,
                               stream_ptr(stream)), "gbk_spmspv")
        return y

    def spmspv_sparse(self, x_ids, x_vals, semiring="lor_land", transpose=False, stream=None):
        """Push SpMSpV with a sparse output: (ids ascending, values) of every reached row."""
        import torch
        n = self.info().ncols if transpose else self.info().nrows
        y_ids = torch.empty(max(n, 1), dtype=torch.int32, device=x_vals.device)
        y_vals = torch.empty(max(n, 1), dtype=x_vals.dtype, device=x_vals.device)
        nv = C.c_int64()
        check(lib().gbk_spmspv_sparse(self.h, int(transpose), SEMIRING[semiring], dtype_code(x_vals), ptr(x_ids),
                                      ptr(x_vals), int(x_ids.numel()), ptr(y_ids), ptr(y_vals), C.byref(nv), None,
                                      stream_ptr(stream)), "gbk_spmspv_sparse")
        return y_ids[:nv.value], y_vals[:nv.value]

    def msbfs(self, sources, levels, direction=0, stream=None):
        """BFS levels from up to 64 sources at once into levels (device int32, len(sources) x n).
        Returns each source's largest level."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        depths = np.zeros(len(src), dtype=np.int32)
        check(lib().gbk_msbfs(self.h, ptr(src), len(src), ptr(levels), int(direction), ptr(depths),
                              stream_ptr(stream)), "gbk_msbfs")
        return depths

    def bfs(self, source, levels, direction=0, stream=None):
        """Single-source BFS levels into levels (device, n elements of int32, int64, float32 or
        float64; source 1, unreached 0).  direction: 0 switches between top-down and bottom-up
        per level, 1 top-down only, 2 bottom-up only.  Returns the largest level."""
        depth = C.c_int32(0)
        check(lib().gbk_bfs_levels(self.h, int(source), int(direction), dtype_code(levels), ptr(levels),
                                   C.byref(depth), stream_ptr(stream)), "gbk_bfs_levels")
        return depth.value

    def sssp(self, source, dist, delta=0.0, stream=None):
        """Shortest-path distances from source into dist (device, n elements of the matrix's value
        type: float32 with FLT_MAX or int32 with INT32_MAX for unreachable).  delta: near-far
        threshold step (0 automatic, < 0 plain worklist).  Returns the rounds run."""
        rounds = C.c_int32(0)
        check(lib().gbk_sssp_dist(self.h, int(source), float(delta), ptr(dist), C.byref(rounds),
                                  stream_ptr(stream)), "gbk_sssp_dist")
        return rounds.value

    def pagerank(self, ranks, itermax=100, damping=0.85, tol=1e-6, stream=None):
        """page_rank_sinks ranks into ranks (device float32, n).  Returns (iterations, last rdiff)."""
        it = C.c_int32(0)
        rd = C.c_float(0)
        check(lib().gbk_pagerank(self.h, int(itermax), float(damping), float(tol), ptr(ranks), C.byref(it),
                                 C.byref(rd), stream_ptr(stream)), "gbk_pagerank")
        return it.value, rd.value

    def pattern_symmetric(self, stream=None) -> bool:
        """True when the matrix equals its transpose in pattern (rows sorted)."""
        out = C.c_int32(0)
        check(lib().gbk_matrix_pattern_symmetric(self.h, C.byref(out), stream_ptr(stream)),
              "gbk_matrix_pattern_symmetric")
        return bool(out.value)

    def cc(self, labels, stream=None):
        """Connected-component labels (smallest vertex id per component) into labels (device, n
        elements of int32, int64 or float32)."""
        check(lib().gbk_cc_labels(self.h, dtype_code(labels), ptr(labels), stream_ptr(stream)), "gbk_cc_labels")

    def ppr(self, seeds, ranks, damping=0.85, tol=1e-6, itermax=100, stream=None):
        """Personalised PageRank for up to 32 seeds into ranks (device float32, len(seeds) x n).
        Returns the iterations each seed ran."""
        src = np.ascontiguousarray(seeds, dtype=np.int32)
        iters = np.zeros(len(src), dtype=np.int32)
        check(lib().gbk_ppr(self.h, ptr(src), len(src), float(damping), float(tol), int(itermax), ptr(ranks),
                            ptr(iters), stream_ptr(stream)), "gbk_ppr")
        return iters

    def sssp_multi(self, sources, dist, stream=None):
        """Integer-weight shortest paths from up to 32 sources into dist (device int32,
        len(sources) x n; INT32_MAX = unreachable).  Returns the rounds each source ran."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        iters = np.zeros(len(src), dtype=np.int32)
        check(lib().gbk_sssp_multi(self.h, ptr(src), len(src), ptr(dist), ptr(iters), stream_ptr(stream)),
              "gbk_sssp_multi")
        return iters

    def batch_autotune(self, kind: str, sources, stream=None) -> BatchTuneResult:
        """Time the batched traversal candidates of `kind` ("bfs", "ppr", "sssp") on these sources
        and keep the fastest for later batched calls and servers on this matrix."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        r = BatchTuneResult()
        check(lib().gbk_batch_autotune(self.h, {"bfs": 0, "ppr": 1, "sssp": 2}[kind], ptr(src), len(src),
                                       C.byref(r), stream_ptr(stream)), "gbk_batch_autotune")
        return r

    def mxm_masked(self, A, B, semiring="plus_one", ctype=I32, stream=None):
        """C<self> = A (+.x) B with this matrix as the mask; returns a new Matrix."""
        out = Matrix.__new__(Matrix)
        out.h = C.c_void_p()
        check(lib().gbk_mxm_masked(C.byref(out.h), self.h, A.h, B.h, SEMIRING[semiring], ctype, stream_ptr(stream)),
              "gbk_mxm_masked")
        out.n, out.ncols, out.nnz, out.vtype = self.n, self.ncols, self.nnz, ctype
        return out


def dense_mask(t, mode="default") -> Mask:
    m = Mask(ptr(t).value, dtype_code(t), MASK[mode], None, 0)
    m._owner = t  # the mask holds a raw pointer: keep its storage alive
    return m


def sparse_mask(ids, mode="default") -> Mask:
    m = Mask(None, 0, MASK[mode], ptr(ids).value, int(ids.numel()))
    m._owner = ids
    return m


def _mp(mask):
    return C.byref(mask) if mask is not None else None


def ewise(op, optype, w, u, v, mask=None, stream=None):
    check(lib().gbk_ewise(BINOP[op], optype, ptr(w), dtype_code(w), ptr(u), dtype_code(u), ptr(v), dtype_code(v),
                          w.numel(), _mp(mask), stream_ptr(stream)), "gbk_ewise")


def apply(kind, op, optype, w, u, scalar=0.0, mask=None, stream=None):
    code = UNOP[op] if kind == 0 else BINOP[op]
    check(lib().gbk_apply(kind, code, optype, ptr(w), dtype_code(w), ptr(u), dtype_code(u), scalar, w.numel(),
                          _mp(mask), stream_ptr(stream)), "gbk_apply")


def assign_scalar(w, value, mask=None, indices=None, stream=None):
    check(lib().gbk_assign_scalar(ptr(w), dtype_code(w), w.numel(), float(value), _mp(mask), ptr(indices),
                                  dtype_code(indices) if indices is not None else I64,
                                  indices.numel() if indices is not None else 0, stream_ptr(stream)),
          "gbk_assign_scalar")


def assign_vector(accum, optype, w, u, mask=None, indices=None, nindices=None, stream=None):
    ni = (indices.numel() if nindices is None else nindices) if indices is not None else 0
    check(lib().gbk_assign_vector(BINOP[accum], optype, ptr(w), dtype_code(w), ptr(u), dtype_code(u), w.numel(),
                                  _mp(mask), ptr(indices), dtype_code(indices) if indices is not None else I64, ni,
                                  stream_ptr(stream)), "gbk_assign_vector")


def extract(accum, optype, w, u, mask=None, indices=None, stream=None):
    check(lib().gbk_extract(BINOP[accum], optype, ptr(w), dtype_code(w), ptr(u), dtype_code(u), w.numel(),
                            _mp(mask), ptr(indices), dtype_code(indices) if indices is not None else I64,
                            indices.numel() if indices is not None else 0, stream_ptr(stream)), "gbk_extract")


def reduce(monoid, rt, u, n=None, stream=None):
    out = {F32: C.c_float, F64: C.c_double, I32: C.c_int32, I64: C.c_int64, BOOL: C.c_uint8}[rt]()
    check(lib().gbk_reduce(MONOID[monoid], rt, ptr(u), dtype_code(u), u.numel() if n is None else n, C.byref(out),
                           stream_ptr(stream)), "gbk_reduce")
    return out.value


def to_sparse(dense, stream=None):
    import torch
    n = dense.numel()
    ids = torch.empty(max(n, 1), dtype=torch.int32, device=dense.device)
    vals = torch.empty(max(n, 1), dtype=dense.dtype, device=dense.device)
    nv = C.c_int64()
    check(lib().gbk_vec_to_sparse(ptr(dense), dtype_code(dense), n, ptr(ids), ptr(vals), C.byref(nv),
                                  stream_ptr(stream)), "gbk_vec_to_sparse")
    return ids[:nv.value], vals[:nv.value]


def to_dense(ids, vals, n, stream=None):
    import torch
    out = torch.empty(n, dtype=vals.dtype, device=vals.device)
    check(lib().gbk_vec_to_dense(ptr(ids), ptr(vals), ids.numel(), dtype_code(vals), ptr(out), n, stream_ptr(stream)),
          "gbk_vec_to_dense")
    return out


def nvals(v, stream=None) -> int:
    out = C.c_int64()
    check(lib().gbk_vec_nvals(ptr(v), dtype_code(v), v.numel(), C.byref(out), stream_ptr(stream)), "gbk_vec_nvals")
    return out.value
