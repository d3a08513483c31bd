// Masked SpGEMM C<M> = A (+.x) B by sorted-list intersection.
//
// Replaces SpMSpM_masked_ikj (src/backend/spmspm/spmspm_masked_hash_based_gustavson.h:9-168),
// which builds a hash set per mask row and a hash map of partial sums.  On
// the GPU every stored (i, j) of the mask is one intersection of row i of A
// with column j of B (both sorted): a warp takes 32 consecutive mask
// entries and, entry by entry, its lanes split the shorter list and binary
// search each element in the longer one, so a hub pair is spread over the
// warp and light pairs cost a few instructions each.
#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

template <int SR, typename C, typename AT>
__global__ void k_masked_spgemm(const int32_t* __restrict__ mptr, const int32_t* __restrict__ midx, int64_t mrows,
                                int64_t mnnz, const int32_t* __restrict__ aptr, const int32_t* __restrict__ aidx,
                                const AT* __restrict__ aval, const int32_t* __restrict__ bptr,
                                const int32_t* __restrict__ bidx, const AT* __restrict__ bval, C* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t groups = (mnnz + 31) / 32;
    for (int64_t g = warp; g < groups; g += nwarps) {
        const int64_t e0 = g * 32;
        // row of the first entry of this group; later entries advance from it
        int64_t lo = 0, hi = mrows;
        while (hi - lo > 1) {
            int64_t mid = (lo + hi) >> 1;
            if (mptr[mid] <= e0)
                lo = mid;
            else
                hi = mid;
        }
        int64_t row = lo;
        const int64_t e_end = min(e0 + 32, mnnz);
        C my_out = C(0);
        for (int64_t e = e0; e < e_end; e++) {
            while (mptr[row + 1] <= e) row++;
            const int32_t j = midx[e];
            int32_t a0 = aptr[row], a1 = aptr[row + 1];
            int32_t b0 = bptr[j], b1 = bptr[j + 1];
            // lanes walk the shorter list, binary-search the longer
            const bool a_short = (a1 - a0) <= (b1 - b0);
            const int32_t s0 = a_short ? a0 : b0, s1 = a_short ? a1 : b1;
            const int32_t l0 = a_short ? b0 : a0, l1 = a_short ? b1 : a1;
            const int32_t* sidx = a_short ? aidx : bidx;
            const int32_t* lidx = a_short ? bidx : aidx;
            C acc = C(0);
            for (int32_t p = s0 + lane; p < s1; p += 32) {
                const int32_t key = sidx[p];
                int32_t lo2 = l0, hi2 = l1;
                while (lo2 < hi2) {
                    int32_t mid = (lo2 + hi2) >> 1;
                    if (lidx[mid] < key)
                        lo2 = mid + 1;
                    else
                        hi2 = mid;
                }
                if (lo2 < l1 && lidx[lo2] == key) {
                    if (SR == GBK_PLUS_ONE) {
                        acc += C(1);
                    } else {
                        const int32_t pa = a_short ? p : lo2;
                        const int32_t pb = a_short ? lo2 : p;
                        acc += C(aval[pa]) * C(bval[pb]);
                    }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
            const C total = __shfl_sync(0xffffffffu, acc, 0);
            if (lane == (int)(e - e0)) my_out = total;
        }
        if (e0 + lane < e_end) out[e0 + lane] = my_out;
    }
}

}  // namespace

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_mxm_masked(gbk_matrix* out, gbk_matrix M, gbk_matrix A, gbk_matrix B, gbk_semiring sr,
                              gbk_dtype ctype, void* stream) {
    GBK_REQUIRE(out && M && A && B, GBK_NULL_POINTER, "gbk_mxm_masked: NULL argument");
    GBK_REQUIRE(sr == GBK_PLUS_ONE || sr == GBK_PLUS_TIMES, GBK_UNSUPPORTED,
                "gbk_mxm_masked: semiring %d not provided (GBK_PLUS_ONE, GBK_PLUS_TIMES)", (int)sr);
    GBK_REQUIRE(ctype == GBK_I32 || ctype == GBK_F32, GBK_UNSUPPORTED, "gbk_mxm_masked: output type %d", (int)ctype);
    GBK_REQUIRE(A->vtype == B->vtype, GBK_DOMAIN_MISMATCH, "gbk_mxm_masked: A and B value types differ");
    GBK_REQUIRE(A->csr.ncols == B->csr.nrows && M->csr.nrows == A->csr.nrows && M->csr.ncols == B->csr.ncols,
                GBK_DIMENSION_MISMATCH, "gbk_mxm_masked: dimensions do not agree");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ensure_csc(B, s);
    if (rc) return rc;
    const CsrView& m = M->csr;
    const CsrView& a = A->csr;
    const CsrView& b = B->csc;
    void* vals = nullptr;
    GBK_CUDA(cudaMalloc(&vals, 4 * (m.nnz > 0 ? m.nnz : 1)));
    if (m.nnz > 0) {
        const int threads = 256;
        int64_t groups = (m.nnz + 31) / 32;
        int64_t blocks = (groups * 32 + threads - 1) / threads;
        int64_t cap = (int64_t)num_sms() * 16;
        if (blocks > cap) blocks = cap;
#define SPGEMM_LAUNCH(SRV, CT, AT)                                                                              \
    k_masked_spgemm<SRV, CT, AT><<<(unsigned)blocks, threads, 0, s>>>(m.ptr, m.idx, m.nrows, m.nnz, a.ptr, a.idx, \
                                                                      (const AT*)a.val, b.ptr, b.idx,           \
                                                                      (const AT*)b.val, (CT*)vals)
        if (A->vtype == GBK_F32) {
            if (sr == GBK_PLUS_ONE) {
                if (ctype == GBK_I32) SPGEMM_LAUNCH(GBK_PLUS_ONE, int32_t, float);
                else SPGEMM_LAUNCH(GBK_PLUS_ONE, float, float);
            } else {
                if (ctype == GBK_I32) SPGEMM_LAUNCH(GBK_PLUS_TIMES, int32_t, float);
                else SPGEMM_LAUNCH(GBK_PLUS_TIMES, float, float);
            }
        } else {
            if (sr == GBK_PLUS_ONE) {
                if (ctype == GBK_I32) SPGEMM_LAUNCH(GBK_PLUS_ONE, int32_t, int32_t);
                else SPGEMM_LAUNCH(GBK_PLUS_ONE, float, int32_t);
            } else {
                if (ctype == GBK_I32) SPGEMM_LAUNCH(GBK_PLUS_TIMES, int32_t, int32_t);
                else SPGEMM_LAUNCH(GBK_PLUS_TIMES, float, int32_t);
            }
        }
#undef SPGEMM_LAUNCH
        GBK_LAUNCHED();
    }
    GBK_CUDA(cudaStreamSynchronize(s));
    rc = gbk_matrix_create_csr(out, m.nrows, m.ncols, m.nnz, m.ptr, m.idx, vals, ctype, 1, stream);
    cudaFree(vals);
    return rc;
}
