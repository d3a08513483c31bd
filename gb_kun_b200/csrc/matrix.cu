// Matrix handles: device CSR, CSC (transpose) and merge-path tiling.
//
// Replaces backend::Matrix<T>::build_from_csr_arrays and csr_to_csc /
// transpose_parallel (src/backend/matrix/build.hpp:170-210,
// src/backend/matrix/transpose.hpp:68-203).  The reference transposes with
// atomic fetch-add cursors, which leaves rows in arbitrary order inside a
// column; here the CSC is produced by a radix sort on (col, row) keys, so
// rows are ascending within each column and every run is deterministic.
#include <algorithm>

#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

__global__ void k_tile_coords(const int32_t* __restrict__ ptr, int64_t nrows, int64_t nnz, int64_t ntiles,
                              int2* __restrict__ coord) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    const int64_t total = nrows + nnz;
    int64_t d = t * (int64_t)kTileItems;
    if (d > total) d = total;
    // smallest i in [lo, hi] with row_end(i) > d - i - 1, row_end(i) = ptr[i + 1]
    int64_t lo = d - nnz > 0 ? d - nnz : 0;
    int64_t hi = d < nrows ? d : nrows;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((int64_t)ptr[mid + 1] <= d - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    coord[t] = make_int2((int)lo, (int)(d - lo));
}

// Row id of every stored entry, by binary search in the row pointers.
__global__ void k_transpose_keys(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, int64_t nrows,
                                 int64_t nnz, unsigned long long* __restrict__ keys, int32_t* __restrict__ pos) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int64_t lo = 0, hi = nrows;  // largest r with ptr[r] <= e
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (ptr[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    keys[e] = ((unsigned long long)(uint32_t)idx[e] << 32) | (uint32_t)lo;
    pos[e] = (int32_t)e;
}

__global__ void k_transpose_finish(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ pos,
                                   const uint32_t* __restrict__ val, int64_t nnz, int32_t* __restrict__ trow,
                                   uint32_t* __restrict__ tval, int32_t* __restrict__ count) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    unsigned long long key = keys[k];
    trow[k] = (int32_t)(key & 0xffffffffULL);
    tval[k] = val[pos[k]];
    warp_count(count, (int32_t)(key >> 32));  // keys sorted by column: one atomic per column per warp
}

int alloc_carries(CsrView& v, int elem_bytes) {
    size_t nt = (size_t)(v.ntiles > 0 ? v.ntiles : 1);
    GBK_CUDA(cudaMalloc(&v.carry_row, nt * sizeof(int32_t)));
    GBK_CUDA(cudaMalloc(&v.carry_val, nt * elem_bytes));
    GBK_CUDA(cudaMalloc(&v.head_val, nt * elem_bytes));
    return GBK_SUCCESS;
}

int bits_for(int64_t n) {
    int b = 1;
    while ((1LL << b) < n) b++;
    return b;
}

}  // namespace

int build_tiles(CsrView& v, int elem_bytes, cudaStream_t s) {
    const int64_t total = v.nrows + v.nnz;
    v.ntiles = (total + kTileItems - 1) / kTileItems;
    GBK_CUDA(cudaMalloc(&v.tile_coord, sizeof(int2) * (v.ntiles + 1)));
    int64_t threads = v.ntiles + 1;
    k_tile_coords<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(v.ptr, v.nrows, v.nnz, v.ntiles, v.tile_coord);
    GBK_LAUNCHED();
    return alloc_carries(v, elem_bytes);
}

void free_view(CsrView& v) {
    cudaFree(v.ptr);
    cudaFree(v.idx);
    cudaFree(v.val);
    cudaFree(v.tile_coord);
    cudaFree(v.carry_row);
    cudaFree(v.carry_val);
    cudaFree(v.head_val);
    free_bins(v.bins);
    free_chunks(v.chunks);
    v = CsrView{};
}

int ensure_csc(gbk_matrix A, cudaStream_t s) {
    if (A->has_csc) return GBK_SUCCESS;
    const CsrView& a = A->csr;
    CsrView& t = A->csc;
    t.nrows = a.ncols;
    t.ncols = a.nrows;
    t.nnz = a.nnz;
    const int64_t nnz = a.nnz;
    const size_t eb = dtype_size(A->vtype);
    GBK_CUDA(cudaMalloc(&t.ptr, sizeof(int32_t) * (t.nrows + 1)));
    GBK_CUDA(cudaMalloc(&t.idx, sizeof(int32_t) * (nnz > 0 ? nnz : 1)));
    GBK_CUDA(cudaMalloc(&t.val, eb * (nnz > 0 ? nnz : 1)));
    GBK_CUDA(cudaMemsetAsync(t.ptr, 0, sizeof(int32_t) * (t.nrows + 1), s));
    if (nnz > 0) {
        // temporaries from the stream-ordered pool (no device-wide
        // synchronisation per allocation or free)
        unsigned long long *keys = nullptr, *keys2 = nullptr;
        int32_t *pos = nullptr, *pos2 = nullptr;
        GBK_CUDA(cudaMallocAsync(&keys, sizeof(unsigned long long) * nnz, s));
        GBK_CUDA(cudaMallocAsync(&keys2, sizeof(unsigned long long) * nnz, s));
        GBK_CUDA(cudaMallocAsync(&pos, sizeof(int32_t) * nnz, s));
        GBK_CUDA(cudaMallocAsync(&pos2, sizeof(int32_t) * nnz, s));
        k_transpose_keys<<<(unsigned)((nnz + 255) / 256), 256, 0, s>>>(a.ptr, a.idx, a.nrows, nnz, keys, pos);
        GBK_LAUNCHED();
        // The entries come in row order, so a stable sort on the column bits
        // alone leaves each column's rows ascending: the low 32 bits (the
        // row) need no passes of their own.
        size_t tmp_bytes = 0;
        const int end_bit = 32 + bits_for(a.ncols + 1);
        cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, pos, pos2, (int)nnz, 32, end_bit, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(tmp_bytes, 16), s));
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, pos, pos2, (int)nnz, 32, end_bit, s));
        count_launch(1);
        // column counts land in ptr[1..], then an inclusive scan gives ptr
        k_transpose_finish<<<(unsigned)((nnz + 255) / 256), 256, 0, s>>>(
            keys2, pos2, (const uint32_t*)a.val, nnz, t.idx, (uint32_t*)t.val, t.ptr + 1);
        GBK_LAUNCHED();
        size_t scan_bytes = 0;
        cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, t.ptr + 1, t.ptr + 1, (int)t.nrows, s);
        void* scan_tmp = nullptr;
        GBK_CUDA(cudaMallocAsync(&scan_tmp, std::max<size_t>(scan_bytes, 16), s));
        GBK_CUDA(cub::DeviceScan::InclusiveSum(scan_tmp, scan_bytes, t.ptr + 1, t.ptr + 1, (int)t.nrows, s));
        count_launch(1);
        for (void* p : {scan_tmp, tmp, (void*)keys, (void*)keys2, (void*)pos, (void*)pos2}) cudaFreeAsync(p, s);
        GBK_CUDA(cudaStreamSynchronize(s));
    }
    int rc = build_tiles(t, (int)eb, s);
    if (rc) return rc;
    t.kernel = A->params.csr_kernel;
    A->has_csc = true;
    return GBK_SUCCESS;
}

}  // namespace gbk

using namespace gbk;

extern "C" {

int gbk_matrix_create_csr(gbk_matrix* out, int64_t nrows, int64_t ncols, int64_t nnz, const int32_t* row_ptr,
                          const int32_t* col, const void* val, gbk_dtype vtype, int on_device, void* stream) {
    GBK_REQUIRE(out, GBK_NULL_POINTER, "gbk_matrix_create_csr: out is NULL");
    GBK_REQUIRE(row_ptr && (nnz == 0 || (col && val)), GBK_NULL_POINTER, "gbk_matrix_create_csr: NULL array");
    GBK_REQUIRE(nrows >= 0 && ncols >= 0 && nnz >= 0, GBK_INVALID_VALUE, "gbk_matrix_create_csr: negative size");
    GBK_REQUIRE(nrows < INT32_MAX && ncols < INT32_MAX && nnz < INT32_MAX, GBK_INVALID_VALUE,
                "gbk_matrix_create_csr: sizes must fit int32 indices (nnz=%lld)", (long long)nnz);
    GBK_REQUIRE(vtype == GBK_F32 || vtype == GBK_I32, GBK_UNSUPPORTED,
                "gbk_matrix_create_csr: matrix values must be GBK_F32 or GBK_I32");
    cudaStream_t s = (cudaStream_t)stream;
    gbk_matrix A = new gbk_matrix_s();
    cudaGetDevice(&A->device);
    A->vtype = vtype;
    CsrView& v = A->csr;
    v.nrows = nrows;
    v.ncols = ncols;
    v.nnz = nnz;
    const size_t eb = dtype_size(vtype);
    auto fail = [&](int rc) {
        free_view(A->csr);
        delete A;
        return rc;
    };
    if (cudaMalloc(&v.ptr, sizeof(int32_t) * (nrows + 1)) != cudaSuccess ||
        cudaMalloc(&v.idx, sizeof(int32_t) * (nnz > 0 ? nnz : 1)) != cudaSuccess ||
        cudaMalloc(&v.val, eb * (nnz > 0 ? nnz : 1)) != cudaSuccess) {
        set_error("gbk_matrix_create_csr: out of device memory (nnz=%lld)", (long long)nnz);
        return fail(GBK_OUT_OF_MEMORY);
    }
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaError_t e = cudaMemcpyAsync(v.ptr, row_ptr, sizeof(int32_t) * (nrows + 1), kind, s);
    if (e == cudaSuccess && nnz > 0) e = cudaMemcpyAsync(v.idx, col, sizeof(int32_t) * nnz, kind, s);
    if (e == cudaSuccess && nnz > 0) e = cudaMemcpyAsync(v.val, val, eb * nnz, kind, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cuda_fail(e, "gbk_matrix_create_csr copy", __FILE__, __LINE__));
    int rc = build_tiles(v, (int)eb, s);
    if (rc) return fail(rc);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cuda_fail(e, "gbk_matrix_create_csr tiles", __FILE__, __LINE__));
    *out = A;
    return GBK_SUCCESS;
}

int gbk_matrix_destroy(gbk_matrix A) {
    if (!A) return GBK_SUCCESS;
    free_batches(A);
    free_single_cache(A);
    free_formats(A);
    free_view(A->csr);
    free_view(A->csc);
    cudaFree(A->xcopy);
    cudaFree(A->coldeg);
    delete A;
    return GBK_SUCCESS;
}

int gbk_matrix_get_info(gbk_matrix A, gbk_matrix_info* info) {
    GBK_REQUIRE(A && info, GBK_NULL_POINTER, "gbk_matrix_get_info: NULL argument");
    info->nrows = A->csr.nrows;
    info->ncols = A->csr.ncols;
    info->nnz = A->csr.nnz;
    info->vtype = A->vtype;
    info->format = A->format;
    info->padded_nnz = format_padded_nnz(A);
    const int64_t eb = (int64_t)dtype_size(A->vtype);
    auto view_bytes = [&](const CsrView& v) {
        if (!v.ptr) return (int64_t)0;
        return (int64_t)(4 * (v.nrows + 1) + (4 + eb) * v.nnz + 8 * (v.ntiles + 1) + (4 + 2 * eb) * v.ntiles);
    };
    info->device_bytes = view_bytes(A->csr) + view_bytes(A->csc) + (int64_t)format_bytes(A);
    info->ntiles = A->csr.ntiles;
    info->has_csc = A->has_csc;
    return GBK_SUCCESS;
}

int gbk_matrix_csr_arrays(gbk_matrix A, int transpose, const int32_t** ptr, const int32_t** idx, const void** val,
                          void* stream) {
    GBK_REQUIRE(A, GBK_NULL_POINTER, "gbk_matrix_csr_arrays: NULL matrix");
    if (transpose) {
        int rc = ensure_csc(A, (cudaStream_t)stream);
        if (rc) return rc;
    }
    const CsrView& v = transpose ? A->csc : A->csr;
    if (ptr) *ptr = v.ptr;
    if (idx) *idx = v.idx;
    if (val) *val = v.val;
    return GBK_SUCCESS;
}

}  // extern "C"
