"""Build recipes for the native libraries (all built in-tree).

* ``gb_kun_b200/libgbk.so``           CUDA kernels + the C ABI (nvcc, sm_100a)
* ``gb_kun_b200/libgbk_graphgen.so``  seeded graph generator (g++ / OpenMP)
* ``gb_kun_b200/libgbk_lablas.so``    C++ lablas:: API + algorithms over the C ABI
* ``oracle/liboracle.so`` and ``oracle/_ref/*``  CPU checkers (test infrastructure)
* ``tests/dropin/_bin/ref_algorithms``  the reference's algorithm files on the
  drop-in header (test infrastructure)

Run ``python -m gb_kun_b200.build`` or call :func:`build_all`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xptxas", "-v"] + ARCH
HOST_CXX = os.environ.get("GBK_CXX", "g++")

# CUDA translation units linked into libgbk.so
CU_SOURCES = [
    "core.cu",
    "matrix.cu",
    "spmv_csr.cu",
    "spmv_bins.cu",
    "spmv_chunks.cu",
    "spmv_formats.cu",
    "spmv_segsmem.cu",
    "spmv_sellw.cu",
    "spmspv.cu",
    "spmspv_sparse.cu",
    "single.cu",
    "vector_ops.cu",
    "spgemm.cu",
    "tune.cu",
    "noalloc.cu",
    "batched.cu",
    "serve.cu",
    "ingest.cu",
]

LABLAS_SOURCES = ["lablas_capi.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, cwd=None, quiet=False):
    res = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(map(str, cmd))}")
    return res.stdout + res.stderr


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_graphgen(force=False) -> Path:
    out = PKG / "libgbk_graphgen.so"
    src = CSRC / "graphgen.cpp"
    if force or _stale(out, [src, INCLUDE / "gbk_graphgen.h"]):
        _run([HOST_CXX, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-march=x86-64-v3",
              "-I", str(INCLUDE), "-o", str(out), str(src)])
    return out


def _headers():
    hs = list(INCLUDE.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    return hs


def build_core(force=False, verbose=False) -> Path:
    out = PKG / "libgbk.so"
    objdir = ROOT / "_build" / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    log = []
    hdrs = _headers()
    for s in CU_SOURCES:
        src = CSRC / s
        if not src.exists():
            continue
        obj = objdir / (src.stem + ".o")
        if force or _stale(obj, [src] + hdrs):
            log.append(_run([nvcc, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src),
                             "-o", str(obj)]))
        objs.append(obj)
    if force or _stale(out, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(out), *map(str, objs), "-lcudart"])
    if verbose:
        print("\n".join(log))
    return out


def build_lablas(force=False) -> Path:
    """C++ lablas:: API and the algorithms, linked against libgbk.so."""
    out = PKG / "libgbk_lablas.so"
    srcs = [CSRC / s for s in LABLAS_SOURCES if (CSRC / s).exists()]
    if not srcs:
        return out
    deps = srcs + list((PKG / "lablas").glob("*.hpp")) + list((PKG / "algorithms").glob("*.hpp")) + \
        list(INCLUDE.glob("*.h")) + [PKG / "libgbk.so"]
    if force or _stale(out, deps):
        cuda = Path(_nvcc()).resolve().parent.parent
        _run([HOST_CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", str(INCLUDE), "-I", str(PKG),
              "-I", str(cuda / "include"), "-o", str(out), *map(str, srcs), "-L", str(PKG), "-lgbk",
              "-L", str(cuda / "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN"])
    return out


def build_oracle(force=False) -> None:
    """CPU checkers: liboracle.so always; the reference harness only where
    the reference sources are present (never on a machine without them)."""
    env = dict(os.environ)
    targets = [str(ROOT / "oracle" / "liboracle.so")]
    # the reference checkout: GBK_REF_DIR, else a "reference" directory beside the repository
    ref_dir = Path(env.get("GBK_REF_DIR", str(ROOT.parent / "reference")))
    env["GBK_REF_DIR"] = str(ref_dir)
    if (ref_dir / "src" / "gb_kun.h").exists():
        targets.append("ref")
    cmd = ["make", "-C", str(ROOT / "oracle")] + (["-B"] if force else []) + targets
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def build_dropin(force=False) -> None:
    """tests/dropin/_bin/ref_algorithms: the reference's own algorithm files,
    unmodified, compiled against the drop-in header (gb_kun_b200/dropin/src)
    and linked with libgbk.so; test infrastructure, built only where the
    reference sources are present."""
    env = dict(os.environ)
    ref_dir = Path(env.get("GBK_REF_DIR", str(ROOT.parent / "reference")))
    if not (ref_dir / "algorithms" / "bfs" / "bfs.hpp").exists():
        return
    env["GBK_REF_DIR"] = str(ref_dir)
    cmd = ["make", "-C", str(ROOT / "tests" / "dropin")] + (["-B"] if force else [])
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def build_all(force=False, verbose=False) -> None:
    build_graphgen(force)
    build_core(force, verbose)
    build_lablas(force)
    build_oracle(force)
    build_dropin(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built")
