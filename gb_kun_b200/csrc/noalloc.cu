// Allocation-free dense -> sparse conversion.
//
// gbk_vec_to_sparse (vector_ops.cu) takes its flag / position arrays and
// the scan's temporary storage from the stream-ordered allocator on every
// call.  Some callers cannot allocate device memory at call time: a host
// framework whose caching allocator has already reserved the free device
// memory (a further cudaMalloc fails), a serving loop that must never wait
// on the allocator in the middle of a request, or an embedding application
// that budgets every byte of device memory before work starts.  This file
// gives them one entry point whose scratch is a fixed file-scope __device__
// array instead.
//
// Scratch: kNoAllocBlocks per-block counts and offsets plus one total
// (about 32 KiB).  Each block owns kNoAllocChunk consecutive entries, so the
// entry point accepts n <= kNoAllocBlocks * kNoAllocChunk = 33,554,432.
// Every GPU that loads this library holds the array until the process exits.
// All calls share it and every slot a call reads is written earlier in the
// same call (nothing has to start at zero); calls that overlap on the GPU
// (different streams, or different host threads without ordering) race on
// it.
//
// Set-up: CUDA loads a module's code and its __device__ arrays lazily, on
// first use, and that load allocates device memory.  gbk_init therefore runs
// noalloc_setup for its device: it looks up the array's device address
// (cudaGetSymbolAddress, with the device current) and queries the three
// kernels (cudaFuncGetAttributes), which loads them, so the array and the
// code are resident before any caller runs out of memory.  The address is
// cached per device.  A device that never saw gbk_init gets the same set-up
// on its first call here (the calls synchronise their stream, so none of
// them is ever inside a stream capture).
// After cudaDeviceReset the module is loaded again and may move: call
// gbk_init again, which refreshes the cached address.
#include <atomic>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocItems = 32;  // entries per thread
constexpr int kNoAllocChunk = kNoAllocThreads * kNoAllocItems;  // 8192 entries per block
constexpr int kNoAllocBlocks = 4096;
constexpr int64_t kNoAllocMaxN = (int64_t)kNoAllocBlocks * kNoAllocChunk;

// [0, kNoAllocBlocks): block counts; [kNoAllocBlocks, 2 kNoAllocBlocks): block
// offsets; [2 kNoAllocBlocks]: total.  Only device code and the set-up below
// use the name; host code passes the address obtained by cudaGetSymbolAddress.
static __device__ __align__(256) int32_t g_noalloc_scratch[2 * kNoAllocBlocks + 1];

__device__ __forceinline__ bool nonzero_at(const void* v, int dt, int64_t i) {
    switch (dt) {
        case GBK_F32: return ((const float*)v)[i] != 0.0f;
        case GBK_I32: return ((const int32_t*)v)[i] != 0;
        case GBK_BOOL: return ((const uint8_t*)v)[i] != 0;
        case GBK_I64: return ((const int64_t*)v)[i] != 0;
        case GBK_F64: return ((const double*)v)[i] != 0.0;
    }
    return false;
}

__device__ __forceinline__ void copy_elem(const void* src, int64_t i, void* dst, int64_t o, int dt) {
    switch (dt) {
        case GBK_F32: ((float*)dst)[o] = ((const float*)src)[i]; break;
        case GBK_I32: ((int32_t*)dst)[o] = ((const int32_t*)src)[i]; break;
        case GBK_BOOL: ((uint8_t*)dst)[o] = ((const uint8_t*)src)[i]; break;
        case GBK_I64: ((int64_t*)dst)[o] = ((const int64_t*)src)[i]; break;
        case GBK_F64: ((double*)dst)[o] = ((const double*)src)[i]; break;
    }
}

// Block-wide exclusive scan of one int per thread (returns the block total).
__device__ int block_exclusive_scan(int v, int* out) {
    __shared__ int warp_sums[kNoAllocThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kNoAllocThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += t;
        }
        if (lane < kNoAllocThreads / 32) warp_sums[lane] = w;  // inclusive warp prefix
    }
    __syncthreads();
    const int warp_prefix = warp > 0 ? warp_sums[warp - 1] : 0;
    *out = warp_prefix + incl - v;
    const int total = warp_sums[kNoAllocThreads / 32 - 1];
    __syncthreads();
    return total;
}

// Pass 1: non-zero count of each block's chunk.
__global__ void __launch_bounds__(kNoAllocThreads) k_na_count(const void* v, int dt, int64_t n, int32_t* scratch) {
    const int64_t base = (int64_t)blockIdx.x * kNoAllocChunk + (int64_t)threadIdx.x * kNoAllocItems;
    int c = 0;
    for (int k = 0; k < kNoAllocItems; k++) {
        const int64_t i = base + k;
        if (i < n && nonzero_at(v, dt, i)) c++;
    }
    int excl;
    const int total = block_exclusive_scan(c, &excl);
    if (threadIdx.x == 0) scratch[blockIdx.x] = total;
}

// Pass 2 (one block): exclusive scan of the block counts, and the total.
__global__ void __launch_bounds__(kNoAllocThreads) k_na_offsets(int nblocks, int32_t* scratch) {
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += kNoAllocThreads) {
        const int b = b0 + threadIdx.x;
        const int c = b < nblocks ? scratch[b] : 0;
        int excl;
        const int total = block_exclusive_scan(c, &excl);
        if (b < nblocks) scratch[kNoAllocBlocks + b] = carry + excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) scratch[2 * kNoAllocBlocks] = carry;
}

// Pass 3: write ids / values at the block offset plus the in-block prefix.
__global__ void __launch_bounds__(kNoAllocThreads) k_na_write(const void* v, int dt, int64_t n,
                                                              const int32_t* scratch, int32_t* ids, void* vals) {
    const int64_t base = (int64_t)blockIdx.x * kNoAllocChunk + (int64_t)threadIdx.x * kNoAllocItems;
    int c = 0;
    for (int k = 0; k < kNoAllocItems; k++) {
        const int64_t i = base + k;
        if (i < n && nonzero_at(v, dt, i)) c++;
    }
    int excl;
    block_exclusive_scan(c, &excl);
    int64_t o = (int64_t)scratch[kNoAllocBlocks + blockIdx.x] + excl;
    for (int k = 0; k < kNoAllocItems; k++) {
        const int64_t i = base + k;
        if (i < n && nonzero_at(v, dt, i)) {
            ids[o] = (int32_t)i;
            copy_elem(v, i, vals, o, dt);
            o++;
        }
    }
}

constexpr int kNoAllocMaxDevices = 64;
std::atomic<int32_t*> g_scratch_addr[kNoAllocMaxDevices];

// Looks up the array's device address for the current device and loads the
// kernels; stores the address in the per-device cache.
int setup_current_device(int dev, int32_t** out) {
    void* p = nullptr;
    GBK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    cudaFuncAttributes fa;
    GBK_CUDA(cudaFuncGetAttributes(&fa, k_na_count));
    GBK_CUDA(cudaFuncGetAttributes(&fa, k_na_offsets));
    GBK_CUDA(cudaFuncGetAttributes(&fa, k_na_write));
    g_scratch_addr[dev].store((int32_t*)p, std::memory_order_release);
    if (out) *out = (int32_t*)p;
    return GBK_SUCCESS;
}

// Device address of the scratch array for the current device.
int scratch_address(int32_t** out) {
    int dev = 0;
    GBK_CUDA(cudaGetDevice(&dev));
    GBK_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, GBK_INVALID_VALUE, "gbk_vec_to_sparse_noalloc: device id %d",
                dev);
    int32_t* a = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (a) {
        *out = a;
        return GBK_SUCCESS;
    }
    return setup_current_device(dev, out);  // two threads racing here store the same address
}

}  // namespace

// Called by gbk_init with `device` current.
int noalloc_setup(int device) {
    GBK_REQUIRE(device >= 0 && device < kNoAllocMaxDevices, GBK_INVALID_VALUE, "gbk_init: device id %d", device);
    return setup_current_device(device, nullptr);
}

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_vec_to_sparse_noalloc(const void* dense, gbk_dtype t, int64_t n, int32_t* ids, void* vals,
                                         int64_t* nvals, void* stream) {
    GBK_REQUIRE(nvals, GBK_NULL_POINTER, "gbk_vec_to_sparse_noalloc: NULL nvals");
    GBK_REQUIRE(n >= 0 && n <= kNoAllocMaxN, GBK_INVALID_VALUE,
                "gbk_vec_to_sparse_noalloc: n = %lld exceeds the fixed scratch limit of %lld entries "
                "(use gbk_vec_to_sparse)",
                (long long)n, (long long)kNoAllocMaxN);
    GBK_REQUIRE(dtype_size(t) > 0, GBK_INVALID_VALUE, "gbk_vec_to_sparse_noalloc: bad type %d", (int)t);
    cudaStream_t s = (cudaStream_t)stream;
    int32_t* scratch = nullptr;
    int rc = scratch_address(&scratch);  // cached by gbk_init, else set up here
    if (rc) return rc;
    if (n == 0) {
        *nvals = 0;
        return GBK_SUCCESS;
    }
    GBK_REQUIRE(dense && ids && vals, GBK_NULL_POINTER, "gbk_vec_to_sparse_noalloc: NULL array");
    const int nblocks = (int)((n + kNoAllocChunk - 1) / kNoAllocChunk);
    k_na_count<<<nblocks, kNoAllocThreads, 0, s>>>(dense, t, n, scratch);
    GBK_LAUNCHED();
    k_na_offsets<<<1, kNoAllocThreads, 0, s>>>(nblocks, scratch);
    GBK_LAUNCHED();
    k_na_write<<<nblocks, kNoAllocThreads, 0, s>>>(dense, t, n, scratch, ids, vals);
    GBK_LAUNCHED();
    int32_t cnt = 0;
    GBK_CUDA(cudaMemcpyAsync(&cnt, scratch + 2 * kNoAllocBlocks, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    *nvals = cnt;
    return GBK_SUCCESS;
}
