"""The reference's own unmasked mxm (SpMSpM_unmasked_ikj) and matrix select,
reached through the harness, against dense numpy: pins the harness wrappers
the GPU tests compare with."""
import numpy as np
import pytest

from gb_kun_b200 import graphgen as gg
from oracle.cpu import Reference

pytestmark = pytest.mark.skipif(not Reference.available(), reason="reference CPU build absent")


def dense(n, rp, col, val):
    A = np.zeros((n, n))
    A[np.repeat(np.arange(n), np.diff(rp)), col] = val
    return A


def test_reference_mxm_is_a_times_a():
    R = Reference()
    g = gg.rmat(9, 4, seed=2)
    val = gg.values_f32(g, seed=1)
    rp, col, v, _ = R.mxm(g, val, 0)
    C = dense(g.n, g.row_ptr, g.col, val) @ dense(g.n, g.row_ptr, g.col, val)
    rows = np.repeat(np.arange(g.n), np.diff(rp))
    assert rp[-1] == np.count_nonzero(C)
    assert np.allclose(C[rows, col], v, rtol=1e-5)


@pytest.mark.parametrize("op,thunk", [(0, -1), (1, 1), (2, 0), (3, 0), (6, 0.5)])
def test_reference_select_keeps_structure(op, thunk):
    R = Reference()
    g = gg.rmat(9, 4, seed=2)
    val = gg.values_f32(g, seed=1)
    rp, col, v = R.select_matrix(g, val, op, thunk)
    assert np.array_equal(rp, g.row_ptr) and np.array_equal(col, g.col)
    i = np.repeat(np.arange(g.n), np.diff(g.row_ptr))
    j = g.col
    keep = {0: j <= i + thunk, 1: j >= i + thunk, 2: j == i + thunk, 3: j != i + thunk, 6: val > thunk}[op]
    assert np.array_equal(v, np.where(keep, val, 0).astype(np.float32))
