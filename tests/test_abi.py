"""The C-ABI libraries load (no GPU needed) and export every entry point
their headers in include/ declare."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
INCLUDE = ROOT / "include"

# header -> library that implements it
HEADERS = {
    "gbk.h": ROOT / "gb_kun_b200" / "libgbk.so",
    "gbk_graphgen.h": ROOT / "gb_kun_b200" / "libgbk_graphgen.so",
    "gbk_lablas.h": ROOT / "gb_kun_b200" / "libgbk_lablas.so",
    "gbk_serve.h": ROOT / "gb_kun_b200" / "libgbk.so",
    "gbk_ingest.h": ROOT / "gb_kun_b200" / "libgbk.so",
}

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**(gbk_[a-z0-9_]+)\s*\(", re.M)


def declared(header: Path):
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(DECL.findall(text)))


@pytest.fixture(scope="module", autouse=True)
def built():
    from gb_kun_b200 import build
    build.build_graphgen()
    build.build_core()
    build.build_lablas()


@pytest.mark.parametrize("header", sorted(HEADERS))
def test_header_symbols_exported(header):
    hpath = INCLUDE / header
    if not hpath.exists():
        pytest.skip(f"{header} not present")
    names = declared(hpath)
    assert names, f"no declarations parsed from {header}"
    lib = C.CDLL(str(HEADERS[header]))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"{HEADERS[header].name} lacks {missing}"


def test_every_header_is_mapped():
    for h in INCLUDE.glob("*.h"):
        if h.name == "gbk_types.h":
            continue
        assert h.name in HEADERS, f"{h.name} has no library mapping in this test"


def test_errors_without_gpu_are_loud():
    """On a machine without an sm_100 device the library reports an error
    instead of computing anything on the CPU."""
    import torch
    from gb_kun_b200 import capi
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(capi.GbkError):
        capi.init(0)
