// Push SpMSpV with a sparse output (the reference's map-based kernels
// spmspv_unmasked_or_map / spmspv_unmasked_critical_map,
// src/backend/spmspv/spmspv_maps.h:5-142, dispatched by the SparseVector
// form of backend::SpMSpV, src/backend/spmspv/spmspv.h:162-205).
//
// The reference collects the reached rows in an std::unordered_map under an
// OpenMP critical section.  Here the frontier's edges are expanded into
// (row, product) pairs -- one thread per edge, its frontier entry found by a
// binary search over the scanned frontier degrees --, sorted by row with a
// stable radix sort (so each row's products keep the frontier / column order),
// and reduced by key with the semiring's add: every reached row appears once,
// ids ascending.  The or-map variant (add probes to 1) stores 1 for every
// reached row, whatever the products, as the reference does.
#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr int kExpThreads = 256;

__global__ void k_sp_degrees(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ids, int64_t nf,
                             int32_t* __restrict__ deg) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < nf) deg[k] = ptr[ids[k] + 1] - ptr[ids[k]];
    if (k == nf) deg[k] = 0;
}

template <int SR, typename T>
__global__ void __launch_bounds__(kExpThreads) k_sp_expand(const int32_t* __restrict__ ptr,
                                                           const int32_t* __restrict__ idx,
                                                           const T* __restrict__ val,
                                                           const int32_t* __restrict__ ids,
                                                           const T* __restrict__ xv, int64_t nf,
                                                           const int32_t* __restrict__ offs, int32_t* __restrict__ key,
                                                           T* __restrict__ prod) {
    using S = Semiring<SR, T>;
    const int64_t E = offs[nf];
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = nf;  // largest k with offs[k] <= e
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (offs[mid] <= e)
                lo = mid;
            else
                hi = mid;
        }
        const int64_t pos = ptr[ids[lo]] + (e - offs[lo]);
        key[e] = idx[pos];
        prod[e] = S::mul(val[pos], xv[lo]);
    }
}

template <int SR, typename T>
struct AddOp {
    __device__ __forceinline__ T operator()(const T& a, const T& b) const { return Semiring<SR, T>::add(a, b); }
};

template <typename T>
__global__ void k_sp_ones(T* __restrict__ v, const int64_t* __restrict__ n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < *n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = T(1);
}

template <int SR, typename T>
int sparse_push(const CsrView& v, const int32_t* ids, const T* xv, int64_t nf, int32_t* y_ids, T* y_vals,
                int64_t* y_nvals, int probe, cudaStream_t s) {
    int32_t *deg = nullptr, *offs = nullptr;
    GBK_CUDA(cudaMallocAsync((void**)&deg, sizeof(int32_t) * (nf + 1), s));
    GBK_CUDA(cudaMallocAsync((void**)&offs, sizeof(int32_t) * (nf + 1), s));
    k_sp_degrees<<<(unsigned)((nf + 1 + 255) / 256), 256, 0, s>>>(v.ptr, ids, nf, deg);
    GBK_LAUNCHED();
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, offs, (int)(nf + 1), s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), s));
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, deg, offs, (int)(nf + 1), s));
    count_launch(1);
    int32_t E32 = 0;
    GBK_CUDA(cudaMemcpyAsync(&E32, offs + nf, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(tmp, s);
    const int64_t E = E32;
    if (E == 0) {
        cudaFreeAsync(deg, s);
        cudaFreeAsync(offs, s);
        *y_nvals = 0;
        return GBK_SUCCESS;
    }
    int32_t *key = nullptr, *key2 = nullptr;
    T *prod = nullptr, *prod2 = nullptr;
    int64_t* nruns = nullptr;
    GBK_CUDA(cudaMallocAsync((void**)&key, 4 * E, s));
    GBK_CUDA(cudaMallocAsync((void**)&key2, 4 * E, s));
    GBK_CUDA(cudaMallocAsync((void**)&prod, sizeof(T) * E, s));
    GBK_CUDA(cudaMallocAsync((void**)&prod2, sizeof(T) * E, s));
    GBK_CUDA(cudaMallocAsync((void**)&nruns, sizeof(int64_t), s));
    const unsigned grid = (unsigned)std::min<int64_t>((E + kExpThreads - 1) / kExpThreads, (int64_t)num_sms() * 16);
    k_sp_expand<SR, T><<<grid, kExpThreads, 0, s>>>(v.ptr, v.idx, (const T*)v.val, ids, xv, nf, offs, key, prod);
    GBK_LAUNCHED();
    int bits = 1;
    while (bits < 31 && (1ll << bits) < v.ncols) ++bits;
    size_t sb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sb, key, key2, prod, prod2, (int)E, 0, bits, s);
    void* stmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&stmp, std::max<size_t>(sb, 16), s));
    GBK_CUDA(cub::DeviceRadixSort::SortPairs(stmp, sb, key, key2, prod, prod2, (int)E, 0, bits, s));
    count_launch(1);
    size_t rb = 0;
    cub::DeviceReduce::ReduceByKey(nullptr, rb, key2, y_ids, prod2, y_vals, nruns, AddOp<SR, T>(), (int)E, s);
    void* rtmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&rtmp, std::max<size_t>(rb, 16), s));
    GBK_CUDA(cub::DeviceReduce::ReduceByKey(rtmp, rb, key2, y_ids, prod2, y_vals, nruns, AddOp<SR, T>(), (int)E, s));
    count_launch(1);
    if (probe == 1) {  // spmspv_unmasked_or_map: every reached row holds 1
        k_sp_ones<T><<<(unsigned)num_sms() * 4, 256, 0, s>>>(y_vals, nruns);
        GBK_LAUNCHED();
    }
    int64_t nr = 0;
    GBK_CUDA(cudaMemcpyAsync(&nr, nruns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    *y_nvals = nr;
    cudaFreeAsync(stmp, s);
    cudaFreeAsync(rtmp, s);
    cudaFreeAsync(key, s);
    cudaFreeAsync(key2, s);
    cudaFreeAsync(prod, s);
    cudaFreeAsync(prod2, s);
    cudaFreeAsync(nruns, s);
    cudaFreeAsync(deg, s);
    cudaFreeAsync(offs, s);
    return GBK_SUCCESS;
}

template <typename T>
int sparse_typed(int sr, const CsrView& v, const int32_t* ids, const T* xv, int64_t nf, int32_t* y_ids, T* y_vals,
                 int64_t* y_nvals, cudaStream_t s) {
    const int probe = semiring_probe(sr, 0);
    switch (sr) {
#define SP_CASE(SRV) \
    case SRV: return sparse_push<SRV, T>(v, ids, xv, nf, y_ids, y_vals, y_nvals, probe, s);
        SP_CASE(GBK_PLUS_TIMES)
        SP_CASE(GBK_LOR_LAND)
        SP_CASE(GBK_FIRST_MIN)
        SP_CASE(GBK_PLUS_SECOND)
        SP_CASE(GBK_STRUCTURAL_BOOL)
        SP_CASE(GBK_MIN_PLUS)
        SP_CASE(GBK_CUSTOM_LESS_PLUS)
        SP_CASE(GBK_MIN_SECOND)
        SP_CASE(GBK_MIN_NOTEQ)
        SP_CASE(GBK_PLUS_ONE)
#undef SP_CASE
        default:
            set_error("gbk_spmspv_sparse: semiring %d has no associative add", sr);
            return GBK_UNSUPPORTED;
    }
}

}  // namespace

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_spmspv_sparse(gbk_matrix A, int transpose, gbk_semiring sr, gbk_dtype dtype, const int32_t* x_ids,
                                 const void* x_vals, int64_t x_nvals, int32_t* y_ids, void* y_vals, int64_t* y_nvals,
                                 const gbk_mask* mask, void* stream) {
    GBK_REQUIRE(A && y_nvals, GBK_NULL_POINTER, "gbk_spmspv_sparse: NULL argument");
    GBK_REQUIRE(x_nvals == 0 || (x_ids && x_vals && y_ids && y_vals), GBK_NULL_POINTER,
                "gbk_spmspv_sparse: NULL frontier or output");
    GBK_REQUIRE(x_nvals >= 0 && x_nvals < INT32_MAX, GBK_INVALID_VALUE, "gbk_spmspv_sparse: bad frontier size");
    GBK_REQUIRE(dtype == A->vtype, GBK_DOMAIN_MISMATCH, "gbk_spmspv_sparse: vector type %d != matrix type %d",
                (int)dtype, (int)A->vtype);
    // spmspv.h:200-204: the reference throws for a mask on the sparse-output form
    GBK_REQUIRE(mask == nullptr, GBK_UNSUPPORTED, "gbk_spmspv_sparse: masked map-based SpMSpV is not provided "
                                                  "(the reference throws for it)");
    cudaStream_t s = (cudaStream_t)stream;
    if (!transpose) {
        int rc = ensure_csc(A, s);
        if (rc) return rc;
    }
    const CsrView& v = transpose ? A->csr : A->csc;
    if (x_nvals == 0) {
        *y_nvals = 0;
        return GBK_SUCCESS;
    }
    if (dtype == GBK_F32)
        return sparse_typed<float>(sr, v, x_ids, (const float*)x_vals, x_nvals, y_ids, (float*)y_vals, y_nvals, s);
    if (dtype == GBK_I32)
        return sparse_typed<int32_t>(sr, v, x_ids, (const int32_t*)x_vals, x_nvals, y_ids, (int32_t*)y_vals, y_nvals,
                                     s);
    set_error("gbk_spmspv_sparse: element type %d unsupported", (int)dtype);
    return GBK_UNSUPPORTED;
}
