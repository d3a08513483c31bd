"""gbk_vec_to_sparse_noalloc: dense -> sparse conversion with no device
allocation at call time.

Callers that cannot allocate device memory when they convert a vector (a
framework whose caching allocator already holds the free memory, a serving
loop that must not wait on the allocator mid-request, an application that
budgets device memory up front) use this entry point; its scratch is a fixed
array inside the library.  The test calls it through the C ABI and checks its
output against the allocating gbk_vec_to_sparse, bit for bit (ids and values
are copied, not computed), on two calls in a row so that the shared scratch
left by the first call cannot leak into the second.  This file is named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MAX_N = 4096 * 8192  # the entry point's documented limit


@pytest.fixture(scope="module")
def capi():
    from gb_kun_b200 import capi
    capi.init(0)
    lib = capi.lib()
    lib.gbk_vec_to_sparse_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p,
                                              C.POINTER(C.c_int64), C.c_void_p]
    lib.gbk_vec_to_sparse_noalloc.restype = C.c_int
    return capi


def noalloc(capi, dense):
    n = dense.numel()
    ids = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    vals = torch.zeros(max(n, 1), dtype=dense.dtype, device="cuda")
    nv = C.c_int64(-1)
    rc = capi.lib().gbk_vec_to_sparse_noalloc(capi.ptr(dense), capi.dtype_code(dense), n, capi.ptr(ids),
                                              capi.ptr(vals), C.byref(nv), capi.stream_ptr())
    capi.check(rc, "gbk_vec_to_sparse_noalloc")
    return ids[:nv.value], vals[:nv.value]


def make(n, density, dtype, seed):
    r = np.random.default_rng(seed)
    x = np.where(r.random(n) < density, r.random(n) * 10 + 1, 0)
    return torch.from_numpy(x.astype(dtype)).cuda()


def pool_state():
    """Reserved and high-water bytes of the device's default stream-ordered
    pool and the device's free memory, read through the CUDA runtime."""
    rt = C.CDLL("libcudart.so.12") if _has("libcudart.so.12") else C.CDLL("libcudart.so")
    dev = C.c_int()
    assert rt.cudaGetDevice(C.byref(dev)) == 0
    pool = C.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    out = []
    for attr in (5, 8):  # cudaMemPoolAttrReservedMemCurrent, cudaMemPoolAttrUsedMemHigh
        v = C.c_uint64()
        assert rt.cudaMemPoolGetAttribute(pool, attr, C.byref(v)) == 0
        out.append(v.value)
    free, _ = torch.cuda.mem_get_info()
    return out[0], out[1], free


def _has(name):
    try:
        C.CDLL(name)
        return True
    except OSError:
        return False


@pytest.mark.parametrize("dtype", [np.float32, np.int32, np.int64, np.float64, np.bool_])
def test_matches_allocating_conversion_twice(capi, dtype):
    # first call: dense vector; second call: a sparser one, so stale scratch would show
    for n, dens, seed in [(3_000_001, 0.4, 1), (1_234_567, 0.001, 2)]:
        d = make(n, dens, dtype, seed)
        ids, vals = noalloc(capi, d)
        ref_ids, ref_vals = capi.to_sparse(d)
        assert ids.numel() == ref_ids.numel()
        assert torch.equal(ids, ref_ids)
        assert torch.equal(vals, ref_vals)


def test_calls_allocate_nothing(capi):
    # inputs and outputs are allocated first; then repeated calls must leave the
    # stream-ordered pool and the device's free memory exactly as they were
    d = make(2_000_003, 0.3, np.float32, 9)
    n = d.numel()
    ids = torch.empty(n, dtype=torch.int32, device="cuda")
    vals = torch.empty(n, dtype=torch.float32, device="cuda")
    nv = C.c_int64(-1)
    fn = capi.lib().gbk_vec_to_sparse_noalloc
    args = (capi.ptr(d), capi.dtype_code(d), n, capi.ptr(ids), capi.ptr(vals), C.byref(nv), capi.stream_ptr())
    capi.check(fn(*args), "gbk_vec_to_sparse_noalloc")
    torch.cuda.synchronize()
    before = pool_state()
    for _ in range(5):
        capi.check(fn(*args), "gbk_vec_to_sparse_noalloc")
    torch.cuda.synchronize()
    after = pool_state()
    assert before == after
    ref_ids, _ = capi.to_sparse(d)
    assert nv.value == ref_ids.numel()


def test_edge_sizes_and_limit(capi):
    for n in (0, 1, 8191, 8192, 8193):
        d = make(n, 0.5, np.float32, n)
        ids, vals = noalloc(capi, d)
        ref_ids, ref_vals = capi.to_sparse(d) if n else (ids, vals)
        assert torch.equal(ids, ref_ids) and torch.equal(vals, ref_vals)
    big = torch.zeros(MAX_N + 1, dtype=torch.uint8, device="cuda")
    with pytest.raises(capi.GbkError) as e:
        noalloc(capi, big)
    assert e.value.status == 5 and "scratch limit" in str(e.value)
