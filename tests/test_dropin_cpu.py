"""The drop-in header compiles for the calls the reference's callers make
(no GPU needed): tests/dropin/api_surface.cpp against
gb_kun_b200/dropin/src/gb_kun.h, syntax only."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def cuda_include():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return str(Path(nvcc).resolve().parent.parent / "include")


def test_dropin_surface_compiles():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    res = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable",
                          "-I", str(ROOT / "gb_kun_b200" / "dropin"), "-I", str(ROOT / "gb_kun_b200"),
                          "-I", str(ROOT / "include"), "-I", cuda_include(),
                          str(ROOT / "tests" / "dropin" / "api_surface.cpp")], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
