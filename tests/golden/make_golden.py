"""Generate the golden fixtures in this folder from the reference's own CPU code.

Runs the reference library (GB_Kun, built from its sources by
``oracle/Makefile`` into ``oracle/_ref/``) on small seeded graphs and stores
inputs and outputs in ``golden.npz``.  Also restates the reference's only
known-answer fixtures (the 6x6 transpose / symmetry cases of
tests/GB_objects/test_matrix_ops.cpp:13-15,131-133) as data.

Run in a container that has the reference sources:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from gb_kun_b200 import graphgen as gg  # noqa: E402
from oracle.cpu import Reference  # noqa: E402

FORMATS = {"CSR": 0, "CSR_SEG": 3, "LAV": 4, "SELL_C": 6}
SEMIRINGS = {"plus_times": 0, "lor_land": 1, "plus_second": 4, "min_plus": 6, "min_second": 8}


def main():
    R = Reference()
    out = {}
    graphs = {
        "rmat10": gg.rmat(10, 16, seed=101),
        "er10": gg.uniform(10, 8, seed=102),
        "rmat11u": gg.rmat(11, 16, seed=103, undirected=True),
        "er11u": gg.uniform(11, 4, seed=104, undirected=True),
    }
    for name, g in graphs.items():
        out[f"{name}.row_ptr"] = g.row_ptr
        out[f"{name}.col"] = g.col
    meta = {"graphs": {"rmat10": [10, 16, 101, 0, "rmat"], "er10": [10, 8, 102, 0, "uniform"],
                       "rmat11u": [11, 16, 103, 1, "rmat"], "er11u": [11, 4, 104, 1, "uniform"]}}

    # SpMV in every storage format and semiring (values and x from the seeded generator)
    for name in ("rmat10", "er10"):
        g = graphs[name]
        val = gg.values_f32(g, seed=201)
        x = gg.vector_f32(g.n, seed=202)
        out[f"{name}.val"] = val
        out[f"{name}.x"] = x
        for fname, fid in FORMATS.items():
            for sname, sid in SEMIRINGS.items():
                y, _ = R.spmv(g, val, x, fmt=fid, semiring=sid)
                out[f"{name}.spmv.{fname}.{sname}"] = y

    # algorithms on the undirected graphs
    for name in ("rmat11u", "er11u"):
        g = graphs[name]
        srcs = gg.sources(g, 3, seed=301)
        out[f"{name}.sources"] = srcs
        for k, s in enumerate(srcs):
            lv, _ = R.bfs(g, int(s))
            out[f"{name}.bfs.{k}"] = lv
        lab, _ = R.cc(g)
        out[f"{name}.cc"] = lab
        w = gg.weights_i32(g, seed=302)
        out[f"{name}.w"] = w
        d, _ = R.sssp(g, w, int(srcs[0]))
        out[f"{name}.sssp"] = d
        for iters in (1, 5, 20):
            r, _ = R.pagerank(g, iters)
            out[f"{name}.pr.{iters}"] = r
        t, _ = R.tc(g)
        out[f"{name}.tc"] = np.array([t], dtype=np.uint64)

    # directed BFS (levels follow out-edges)
    g = graphs["rmat10"]
    srcs = gg.sources(g, 2, seed=303)
    out["rmat10.sources"] = srcs
    for k, s in enumerate(srcs):
        lv, _ = R.bfs(g, int(s))
        out[f"rmat10.bfs.{k}"] = lv

    # known-answer fixtures restated from tests/GB_objects/test_matrix_ops.cpp
    meta["transpose_kat"] = {
        "rows": [0, 0, 1, 1, 1, 2, 3, 4, 5],
        "cols": [2, 4, 0, 3, 5, 1, 4, 2, 0],
        "expected_csc_sets": [[1, 5], [2], [0, 4], [1], [0, 3], [1]],
    }
    meta["symmetric_kat"] = {"rows": [0, 0, 1, 2, 2, 3, 4, 4, 5], "cols": [1, 3, 0, 2, 4, 0, 2, 5, 4]}

    # The reference's CSR SpMV splits rows over OpenMP threads by nnz and
    # skips trailing empty rows when nnz is a multiple of the thread count
    # (src/helpers/balancing/balancing.h:12-22); the checker needs that count.
    meta["omp_threads"] = R.max_threads()
    np.savez_compressed(HERE / "golden.npz", **out)
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1))
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
