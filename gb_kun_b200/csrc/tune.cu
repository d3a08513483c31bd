// Per-graph autotuner: times every storage format / CSR kernel candidate for
// the matrix at hand and keeps the fastest.  The reference picks its format
// from the command line (-format, src/helpers/cmd_parser/cmd_parser.hpp) and
// fixes C / sigma at compile time (la_backend.h:16-34); here the choice is
// measured on the device.  Results are cached per graph fingerprint (shape,
// nnz and a log2 degree histogram) for the life of the process, and in the
// text file named by GBK_TUNE_CACHE when that variable is set.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

struct Candidate {
    gbk_format fmt;
    int32_t sigma;
    int32_t kernel;
    int32_t hot;
    int32_t staged;  // SELL-C: 1 = inside staged x windows (hot == -1 then renumbers the columns first)
};

// Order matches gbk_tune_result.candidate_ms (include/gbk.h).
const Candidate kCandidates[] = {
    {GBK_FMT_CSR, 0, kKernelBins, 0},        {GBK_FMT_CSR, 0, kKernelMerge, 0},
    {GBK_FMT_SELL_C, 1, kKernelAuto, 0},     {GBK_FMT_SELL_C, 256, kKernelAuto, 0},
    {GBK_FMT_SELL_C, 4096, kKernelAuto, 0},  {GBK_FMT_CSR_SEG, 0, kKernelAuto, 0},
    {GBK_FMT_LAV, 0, kKernelAuto, 0},        {GBK_FMT_SELL_C, 4096, kKernelAuto, 16384},
    {GBK_FMT_SELL_C, 4096, kKernelAuto, 53248}, {GBK_FMT_SELL_C, 256, kKernelAuto, 53248},
    {GBK_FMT_SELL_C, 4096, kKernelAuto, -1},    {GBK_FMT_SELL_C, 256, kKernelAuto, -1},
    {GBK_FMT_SELL_C, 0, kKernelAuto, 0, 1},     {GBK_FMT_SELL_C, 0, kKernelAuto, -1, 1},
    {GBK_FMT_CSR, 0, kKernelChunks, 0},
};
constexpr int kNumCandidates = sizeof(kCandidates) / sizeof(kCandidates[0]);

std::mutex g_mu;
std::map<std::string, int> g_cache;
bool g_file_loaded = false;

int fingerprint(gbk_matrix A, int transpose, int sr, std::string* out, cudaStream_t s) {
    const CsrView& v = transpose ? A->csc : A->csr;
    std::vector<int32_t> p(v.nrows + 1);
    GBK_CUDA(cudaMemcpyAsync(p.data(), v.ptr, 4 * (v.nrows + 1), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    int64_t hist[33] = {0};
    for (int64_t i = 0; i < v.nrows; i++) {
        int d = p[i + 1] - p[i], b = 0;
        while (d) {
            b++;
            d >>= 1;
        }
        hist[b]++;
    }
    char buf[64];
    std::string f = std::to_string(v.nrows) + "x" + std::to_string(v.ncols) + ":" + std::to_string(v.nnz) + ":t" +
                    std::to_string(transpose) + ":sr" + std::to_string(sr) + ":v" + std::to_string((int)A->vtype);
    for (int b = 0; b < 33; b++) {
        std::snprintf(buf, sizeof(buf), ":%lld", (long long)hist[b]);
        f += buf;
    }
    *out = f;
    return GBK_SUCCESS;
}

void load_file_cache() {
    if (g_file_loaded) return;
    g_file_loaded = true;
    const char* path = std::getenv("GBK_TUNE_CACHE");
    if (!path) return;
    FILE* fp = std::fopen(path, "r");
    if (!fp) return;
    char key[2048];
    int idx;
    while (std::fscanf(fp, "%2047s %d", key, &idx) == 2)
        if (idx >= 0 && idx < kNumCandidates) g_cache[key] = idx;
    std::fclose(fp);
}

void store_file_cache(const std::string& key, int idx) {
    const char* path = std::getenv("GBK_TUNE_CACHE");
    if (!path) return;
    FILE* fp = std::fopen(path, "a");
    if (!fp) return;
    std::fprintf(fp, "%s %d\n", key.c_str(), idx);
    std::fclose(fp);
}

template <typename T>
__global__ void k_fill_ones(T* x, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) x[i] = T(1);
}

int apply_candidate(gbk_matrix A, const Candidate& c, cudaStream_t s) {
    gbk_format_params p = A->params;
    p.sell_sigma = c.sigma ? c.sigma : 4096;
    p.csr_kernel = c.kernel;
    p.sell_hot_cols = c.hot > 0 ? c.hot : 0;
    p.sell_reorder_cols = c.hot < 0 ? 1 : 0;  // hot == -1: renumbered columns
    if (c.fmt == GBK_FMT_SELL_C) p.seg_staged = c.staged;
    else if (p.seg_staged > 0) p.seg_staged = 0;
    return build_format(A, c.fmt, &p, s);
}

}  // namespace

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_matrix_autotune(gbk_matrix A, int transpose, gbk_semiring sr, int32_t reps,
                                   gbk_tune_result* result, void* stream) {
    GBK_REQUIRE(A, GBK_NULL_POINTER, "gbk_matrix_autotune: NULL matrix");
    cudaStream_t s = (cudaStream_t)stream;
    if (reps <= 0) reps = 20;
    int rc = ensure_csc(A, s);
    if (rc) return rc;
    std::string key;
    rc = fingerprint(A, transpose, sr, &key, s);
    if (rc) return rc;
    gbk_tune_result res{};
    res.ncandidates = kNumCandidates;
    int best = -1;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_file_cache();
        auto it = g_cache.find(key);
        if (it != g_cache.end()) best = it->second;
    }
    if (best >= 0) {
        res.cached = 1;
    } else {
        const CsrView& v = transpose ? A->csc : A->csr;
        const size_t eb = dtype_size(A->vtype);
        void *x = nullptr, *y = nullptr;
        GBK_CUDA(cudaMalloc(&x, eb * (v.ncols > 0 ? v.ncols : 1)));
        GBK_CUDA(cudaMalloc(&y, eb * (v.nrows > 0 ? v.nrows : 1)));
        if (v.ncols > 0) {
            if (A->vtype == GBK_F32)
                k_fill_ones<float><<<(unsigned)((v.ncols + 255) / 256), 256, 0, s>>>((float*)x, v.ncols);
            else
                k_fill_ones<int32_t><<<(unsigned)((v.ncols + 255) / 256), 256, 0, s>>>((int32_t*)x, v.ncols);
            GBK_LAUNCHED();
        }
        cudaEvent_t e0, e1;
        GBK_CUDA(cudaEventCreate(&e0));
        GBK_CUDA(cudaEventCreate(&e1));
        float best_ms = 1e30f;
        for (int c = 0; c < kNumCandidates; c++) {
            rc = apply_candidate(A, kCandidates[c], s);
            if (rc) break;
            for (int w = 0; w < 3 && !rc; w++)
                rc = gbk_mxv(A, transpose, sr, GBK_OP_SECOND, A->vtype, x, y, nullptr, GBK_BOOL, GBK_MASK_DEFAULT, s);
            GBK_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < reps && !rc; r++)
                rc = gbk_mxv(A, transpose, sr, GBK_OP_SECOND, A->vtype, x, y, nullptr, GBK_BOOL, GBK_MASK_DEFAULT, s);
            GBK_CUDA(cudaEventRecord(e1, s));
            GBK_CUDA(cudaEventSynchronize(e1));
            if (rc) break;
            float ms = 0;
            GBK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms /= reps;
            res.candidate_ms[c] = ms;
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(x);
        cudaFree(y);
        if (rc) return rc;
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[key] = best;
        store_file_cache(key, best);
    }
    rc = apply_candidate(A, kCandidates[best], s);
    if (rc) return rc;
    res.format = kCandidates[best].fmt;
    res.sell_sigma = kCandidates[best].sigma;
    res.csr_kernel = kCandidates[best].kernel;
    res.sell_hot_cols = kCandidates[best].hot;  // -1: columns renumbered
    res.sell_staged = kCandidates[best].staged;
    res.best_ms = res.cached ? 0.0f : res.candidate_ms[best];
    if (result) *result = res;
    return GBK_SUCCESS;
}
