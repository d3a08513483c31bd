import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"

# Tolerance for FP32 results against the FP64 oracle (relative L1 norm).
REL_L1_TOL = 1e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


def rel_l1(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def golden():
    data = np.load(GOLDEN / "golden.npz")
    meta = json.loads((GOLDEN / "golden.json").read_text())
    return data, meta


@pytest.fixture(scope="session")
def oracle():
    from oracle.cpu import Oracle
    return Oracle()


def golden_graph(data, name):
    from gb_kun_b200.graphgen import Graph
    rp = data[f"{name}.row_ptr"]
    return Graph(n=len(rp) - 1, row_ptr=rp, col=data[f"{name}.col"], name=name)
