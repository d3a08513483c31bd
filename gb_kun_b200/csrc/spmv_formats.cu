// Optimised storage formats (SELL-C-sigma, segmented CSR, LAV).
#include "common.cuh"
#include "internal.h"

namespace gbk {

int spmv_format(gbk_matrix A, int transpose, int sr, int accum, int dtype, const void* x, void* y,
                cudaStream_t s) {
    const CsrView& v = transpose ? A->csc : A->csr;
    return spmv_csr(v, sr, accum, dtype, x, y, nullptr, 0, 0, s);
}

int build_format(gbk_matrix A, gbk_format fmt, const gbk_format_params* p, cudaStream_t s) {
    (void)p;
    (void)s;
    if (fmt == GBK_FMT_CSR) {
        A->format = fmt;
        return GBK_SUCCESS;
    }
    set_error("format %d not built yet", (int)fmt);
    return GBK_UNSUPPORTED;
}

size_t format_bytes(gbk_matrix A) { return 0; }
int64_t format_padded_nnz(gbk_matrix A) { return A->csr.nnz; }
int free_formats(gbk_matrix A) { return GBK_SUCCESS; }

}  // namespace gbk

extern "C" int gbk_matrix_set_format(gbk_matrix A, gbk_format fmt, const gbk_format_params* params, void* stream) {
    GBK_REQUIRE(A, GBK_NULL_POINTER, "gbk_matrix_set_format: NULL matrix");
    return gbk::build_format(A, fmt, params, (cudaStream_t)stream);
}
