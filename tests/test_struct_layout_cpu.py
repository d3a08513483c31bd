"""The ctypes mirrors of the C-ABI structs (gb_kun_b200/capi.py, serve.py,
graphgen.py) have the size and field offsets that a C compiler gives the
structs in include/*.h.  A field added to a header but not to its mirror (or
reordered) would otherwise pass garbage across the boundary without an error.
Compiles one small C program with gcc; no GPU needed."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
INCLUDE = ROOT / "include"


def mirrors():
    from gb_kun_b200 import capi, graphgen, serve
    return [
        ("gbk_format_params", "gbk.h", capi.FormatParams),
        ("gbk_mask", "gbk.h", capi.Mask),
        ("gbk_matrix_info", "gbk.h", capi.MatrixInfo),
        ("gbk_tune_result", "gbk.h", capi.TuneResult),
        ("gbk_batch_tune_result", "gbk.h", capi.BatchTuneResult),
        ("gbk_file_info", "gbk_ingest.h", capi.FileInfo),
        ("gbk_graph", "gbk_graphgen.h", graphgen._GbkGraph),
        ("gbk_server_config", "gbk_serve.h", serve.ServerConfig),
        ("gbk_query_result", "gbk_serve.h", serve.QueryResult),
    ]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    ms = mirrors()
    headers = sorted({h for _, h, _ in ms})
    lines = ["#include <stdio.h>", "#include <stddef.h>"] + [f'#include "{h}"' for h in headers]
    lines.append("int main(void) {")
    for cname, _, cls in ms:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    d = tmp_path_factory.mktemp("layout")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-I", str(INCLUDE), str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        struct, field, value = line.split()
        table[(struct, field)] = int(value)
    return table


@pytest.mark.parametrize("idx", range(9))
def test_ctypes_mirror_matches_header(c_layout, idx):
    cname, _, cls = mirrors()[idx]
    assert C.sizeof(cls) == c_layout[(cname, "sizeof")], cname
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == c_layout[(cname, fname)], (cname, fname)
