// Internal (non-ABI) declarations shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "gbk.h"

namespace gbk {

// Merge-path tiling of one CSR orientation: tile t covers merge diagonals
// [t * kTileItems, (t + 1) * kTileItems) of the merged (row-end, nnz) list.
constexpr int kSpmvThreads = 256;
constexpr int kSpmvItems = 8;
constexpr int kTileItems = kSpmvThreads * kSpmvItems;

struct RowBins;    // spmv_bins.cu
struct RowChunks;  // spmv_chunks.cu

// CSR kernel choice of a view: degree-binned lane groups, merge-path tiles or
// equal runs of 256 entries per warp.
enum { kKernelAuto = 0, kKernelMerge = 1, kKernelBins = 2, kKernelChunks = 3 };

struct CsrView {
    int64_t nrows = 0, ncols = 0, nnz = 0;
    int kernel = kKernelAuto;
    mutable RowBins* bins = nullptr;      // built on first use
    mutable RowChunks* chunks = nullptr;  // built on first use
    int32_t* ptr = nullptr;  // nrows + 1
    int32_t* idx = nullptr;  // nnz
    void* val = nullptr;     // nnz of the matrix value type
    // merge-path tiles
    int64_t ntiles = 0;
    int2* tile_coord = nullptr;  // ntiles + 1 (row, nnz) start coordinates
    // per-tile carries for rows that cross tiles (scratch, kept with the view)
    int32_t* carry_row = nullptr;  // ntiles
    void* carry_val = nullptr;     // ntiles elements (4 bytes each)
    void* head_val = nullptr;      // ntiles elements
};

struct SellC;     // spmv_formats.cu
struct SegCsr;    // spmv_formats.cu (CSR_SEG and LAV share one layout)
struct SegSmem;   // spmv_segsmem.cu (CSR_SEG with x windows staged in shared memory)
struct SingleCache;  // single.cu
struct SellW;     // spmv_sellw.cu (SELL-C-sigma inside x windows staged in shared memory)
struct Batch;     // batched.h

// Tunables of the batched traversals (batched.cu).
struct BatchOptions {
    int bfs_direction = 0;    // 0 = auto, 1 = push only, 2 = pull only
    int bfs_alpha = 4;        // switch to pull when frontier edges * alpha > unvisited edges
    int bfs_beta = 24;        // switch back to push when frontier vertices * beta < n
    int item_edges = 256;     // PPR / SSSP: edges per warp work item
    float damping = 0.85f;    // PPR
    double tol = 1e-6;        // PPR: stop when sum |r_new - r_old| < tol
    int itermax = 100;        // PPR iteration cap
    int sssp_max_iter = 0;    // SSSP iteration cap (0: n)
};

}  // namespace gbk

struct gbk_matrix_s {
    gbk_dtype vtype = GBK_F32;
    gbk::CsrView csr;           // A
    gbk::CsrView csc;           // A^T (built lazily)
    bool has_csc = false;
    int8_t pattern_symmetric = -1;  // -1 unknown; gbk_matrix_pattern_symmetric
    int32_t* coldeg = nullptr;      // entries per column, built by the first gbk_pagerank
    int64_t coldeg_zero = 0;        // columns without entries (valid with coldeg)
    gbk::SingleCache* single = nullptr;  // scratch and graphs of the single-query loops
    int64_t format_gen = 0;         // bumped whenever the storage format changes
    gbk_format format = GBK_FMT_CSR;
    gbk_format_params params{};
    gbk::SellC* sell[2] = {nullptr, nullptr};
    gbk::SegCsr* seg[2] = {nullptr, nullptr};
    gbk::SegCsr* lav[2] = {nullptr, nullptr};
    gbk::SegSmem* segx[2] = {nullptr, nullptr};
    gbk::SellW* sellw[2] = {nullptr, nullptr};
    void* xcopy = nullptr;      // n elements, used when x aliases y
    int64_t xcopy_elems = 0;
    int device = 0;
    // batches kept for the one-shot batched calls (BFS, PPR, SSSP)
    gbk::Batch* batch[3] = {nullptr, nullptr, nullptr};
    gbk::BatchOptions batch_opt[3];
    // options chosen by gbk_batch_autotune, per kind
    bool batch_tuned[3] = {false, false, false};
    gbk::BatchOptions batch_tuned_opt[3];
};

namespace gbk {

int build_bins(const CsrView& v, int elem_bytes, RowBins** out, cudaStream_t s);
void free_bins(RowBins* b);
bool chunks_usable(const CsrView& v);
int build_chunks(const CsrView& v, int elem_bytes, RowChunks** out, cudaStream_t s);
void free_chunks(RowChunks* c);
int spmv_chunks(const RowChunks* rc, const CsrView& v, int sr, int accum, int dtype, const void* x, void* y,
                const void* mask, int mdt, int mmode, cudaStream_t s);
int spmv_binned(const RowBins* rb, const CsrView& v, int sr, int accum, int dtype, const void* x, void* y,
                const void* mask, int mdt, int mmode, cudaStream_t s);

int ensure_csc(gbk_matrix A, cudaStream_t s);
void free_single_cache(gbk_matrix A);
void free_batches(gbk_matrix A);  // batched.cu
int build_tiles(CsrView& v, int elem_bytes, cudaStream_t s);
void free_view(CsrView& v);
int free_formats(gbk_matrix A);

// SpMV on one CSR orientation (merge-path); y = accum(y, A x) with optional
// dense mask.  Defined in spmv_csr.cu.
int spmv_csr(const CsrView& v, int sr, int accum, int dtype, const void* x, void* y, const void* mask,
             int mask_dtype, int mask_mode, cudaStream_t s);

// Storage-format SpMV (unmasked), defined in spmv_formats.cu.
int spmv_format(gbk_matrix A, int transpose, int sr, int accum, int dtype, const void* x, void* y,
                cudaStream_t s);
int build_format(gbk_matrix A, gbk_format fmt, const gbk_format_params* p, cudaStream_t s);
size_t format_bytes(gbk_matrix A);

// CSR_SEG with staged x windows (spmv_segsmem.cu).  run_segsmem returns
// GBK_UNSUPPORTED for semirings whose add it cannot fold atomically.
int build_segsmem(const CsrView& a, int dtype, SegSmem** out, cudaStream_t s);
int run_segsmem(const SegSmem* f, int sr, int accum, int dtype, const void* x, void* y, cudaStream_t s);
void free_segsmem(SegSmem* f);
size_t segsmem_bytes(const SegSmem* f);
int64_t format_padded_nnz(gbk_matrix A);
// SELL-C-sigma inside staged x windows (spmv_sellw.cu); run_sellw returns
// GBK_UNSUPPORTED for semirings whose add it cannot fold atomically.
int build_sellw(const CsrView& a, int dtype, bool reorder, SellW** out, cudaStream_t s);
int run_sellw(const SellW* f, int sr, int accum, int dtype, const void* x, void* y, cudaStream_t s);
void free_sellw(SellW* f);
size_t sellw_bytes(const SellW* f);
int64_t sellw_padded(const SellW* f);
// Column order by in-degree (spmv_formats.cu): new_to_old and relabelled
// column ids, both cudaMalloc'd for the caller.
int indegree_order(const CsrView& a, float dense_frac, int32_t** new_to_old, int32_t** idx_out,
                   int64_t* dense_cols, cudaStream_t s);

}  // namespace gbk
