// CSR SpMV by degree bins: one launch, no shared memory, no barriers.
//
// Rows are grouped by degree at build time (a stable sort by bin keeps rows
// ascending inside a bin):
//   bin 0           empty rows                      one thread per row
//   bins G=1..32    degree in (G/2, G]              G lanes per row (shuffle reduce)
//   warp bin        degree 33..kSplitNnz            one warp per row, 4 loads in flight per lane
//   split bin       degree > kSplitNnz              the row is cut into kSplitNnz chunks,
//                                                   one warp per chunk, partials folded
//                                                   in chunk order by a small fix-up kernel
// A block table maps every CTA of the single grid to its bin, so the whole
// SpMV is two launches whatever the degree distribution.  The heaviest bins
// take the lowest CTA ids (split chunks, then warp rows, then the lane groups
// from 32 down): CTAs start roughly in id order, so the longest work starts
// first instead of in the grid's last wave.  Each group streams
// its rows' col / val once (coalesced inside a row) and gathers x through L2.
// This is the same computation as SpMV_all_active_diff_vectors
// (src/backend/spmv/spmv_csr.h:340-384) with the reference's nnz-balanced
// thread ranges (src/helpers/balancing/balancing.h:5-33) replaced by
// degree-matched lane groups.
#include <cub/cub.cuh>

#include <vector>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr int kBinThreads = 256;
#ifndef GBK_SPLIT_NNZ
#define GBK_SPLIT_NNZ 2048
#endif
constexpr int kSplitNnz = GBK_SPLIT_NNZ;
// bins: 0 empty, 1..6 -> G = 1,2,4,8,16,32, 7 warp, 8 split
constexpr int kNumBins = 9;
constexpr int kBinWarp = 7;
constexpr int kBinSplit = 8;

__host__ __device__ inline int bin_of_degree(int d) {
    if (d == 0) return 0;
    if (d <= 1) return 1;
    if (d <= 2) return 2;
    if (d <= 4) return 3;
    if (d <= 8) return 4;
    if (d <= 16) return 5;
    if (d <= 32) return 6;
    if (d <= kSplitNnz) return kBinWarp;
    return kBinSplit;
}

struct BinTable {
    int32_t block_start[kNumBins];      // CTA range [block_start, block_end) per bin
    int32_t block_end[kNumBins];
    int32_t item_start[kNumBins];       // first item of the bin in perm (split bin: chunk table)
    int32_t items[kNumBins];            // rows (or chunks) in the bin
};

template <typename T>
__device__ __forceinline__ void write_out(T* y, int64_t r, T v, int accum, const void* mask, int mdt, int mmode) {
    if (mask && !mask_selects(mask, mdt, mmode, r)) {
        y[r] = T(0);
        return;
    }
    y[r] = (accum == GBK_OP_SECOND) ? v : binop<T>(accum, y[r], v);
}

template <int SR, typename T, int G>
__device__ __forceinline__ void rows_by_group(const BinTable& bt, int bin, int lb, const int32_t* __restrict__ ptr,
                                              const int32_t* __restrict__ idx, const T* __restrict__ val,
                                              const int32_t* __restrict__ perm, const T* __restrict__ x,
                                              T* __restrict__ y, int accum, const void* mask, int mdt, int mmode) {
    using S = Semiring<SR, T>;
    const int sub = threadIdx.x % G;
    const int64_t k = (int64_t)lb * (kBinThreads / G) + threadIdx.x / G;
    const bool live = k < bt.items[bin];
    int32_t r = 0;
    T acc = S::identity();
    bool skip = !live;
    if (live) {
        r = perm[bt.item_start[bin] + k];
        if (mask && !mask_selects(mask, mdt, mmode, r)) skip = true;
        if (!skip) {
            const uint64_t pol = policy_evict_last();
            const int32_t b = ld_stream(ptr + r), e = ld_stream(ptr + r + 1);
            for (int32_t q = b + sub; q < e; q += G)
                acc = S::add(acc, S::mul(ld_stream(val + q), ld_keep(x + ld_stream(idx + q), pol)));
        }
    }
    if (G > 1) {
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) acc = S::add(acc, __shfl_xor_sync(0xffffffffu, acc, off, G));
    }
    if (live && sub == 0) {
        if (skip)
            y[r] = T(0);  // outside the mask (spmv_csr.h:324-327)
        else
            y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
    }
}

template <int SR, typename T>
__device__ __forceinline__ T warp_range(int32_t b, int32_t e, const int32_t* __restrict__ idx,
                                        const T* __restrict__ val, const T* __restrict__ x, int lane) {
    using S = Semiring<SR, T>;
    // software-pipelined: the next U groups of 32 entries are loaded before
    // the x values of the current groups are gathered
    constexpr int U = 4;
    const uint64_t pol = policy_evict_last();
    T acc = S::identity();
    int c[U];
    T a[U];
    int32_t q = b + lane;
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int32_t p = q + 32 * u;
        c[u] = p < e ? ld_stream(idx + p) : -1;
        a[u] = p < e ? ld_stream(val + p) : T(0);
    }
    for (; q < e; q += 32 * U) {
        int cn[U];
        T an[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int32_t p = q + 32 * (U + u);
            cn[u] = p < e ? ld_stream(idx + p) : -1;
            an[u] = p < e ? ld_stream(val + p) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (c[u] >= 0) acc = S::add(acc, S::mul(a[u], ld_keep(x + c[u], pol)));
#pragma unroll
        for (int u = 0; u < U; u++) {
            c[u] = cn[u];
            a[u] = an[u];
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc = S::add(acc, __shfl_xor_sync(0xffffffffu, acc, off));
    return acc;
}

template <int SR, typename T>
__global__ void __launch_bounds__(kBinThreads) k_spmv_binned(
    BinTable bt, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val,
    const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk_row, const int32_t* __restrict__ chunk_beg,
    const T* __restrict__ x, T* __restrict__ y, int accum, const void* mask, int mdt, int mmode,
    T* __restrict__ chunk_out) {
    using S = Semiring<SR, T>;
    int bin = 0;
#pragma unroll
    for (int b = 1; b < kNumBins; b++)
        if ((int)blockIdx.x >= bt.block_start[b] && (int)blockIdx.x < bt.block_end[b]) bin = b;
    const int lb = blockIdx.x - bt.block_start[bin];
    switch (bin) {
        case 0: {  // empty rows: the identity, accumulated
            const int64_t k = (int64_t)lb * kBinThreads + threadIdx.x;
            if (k < bt.items[0]) write_out<T>(y, perm[bt.item_start[0] + k], S::identity(), accum, mask, mdt, mmode);
            return;
        }
        case 1: rows_by_group<SR, T, 1>(bt, 1, lb, ptr, idx, val, perm, x, y, accum, mask, mdt, mmode); return;
        case 2: rows_by_group<SR, T, 2>(bt, 2, lb, ptr, idx, val, perm, x, y, accum, mask, mdt, mmode); return;
        case 3: rows_by_group<SR, T, 4>(bt, 3, lb, ptr, idx, val, perm, x, y, accum, mask, mdt, mmode); return;
        case 4: rows_by_group<SR, T, 8>(bt, 4, lb, ptr, idx, val, perm, x, y, accum, mask, mdt, mmode); return;
        case 5: rows_by_group<SR, T, 16>(bt, 5, lb, ptr, idx, val, perm, x, y, accum, mask, mdt, mmode); return;
        case 6: rows_by_group<SR, T, 32>(bt, 6, lb, ptr, idx, val, perm, x, y, accum, mask, mdt, mmode); return;
        case kBinWarp: {
            const int lane = threadIdx.x & 31;
            const int64_t k = (int64_t)lb * (kBinThreads / 32) + (threadIdx.x >> 5);
            if (k >= bt.items[kBinWarp]) return;
            const int32_t r = perm[bt.item_start[kBinWarp] + k];
            if (mask && !mask_selects(mask, mdt, mmode, r)) {
                if (lane == 0) y[r] = T(0);
                return;
            }
            T acc = warp_range<SR, T>(ptr[r], ptr[r + 1], idx, val, x, lane);
            if (lane == 0) y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
            return;
        }
        default: {  // split rows: one chunk per warp
            const int lane = threadIdx.x & 31;
            const int64_t k = (int64_t)lb * (kBinThreads / 32) + (threadIdx.x >> 5);
            if (k >= bt.items[kBinSplit]) return;
            const int32_t r = chunk_row[k];
            const int32_t b = chunk_beg[k];
            const int32_t e = min(b + kSplitNnz, ptr[r + 1]);
            if (mask && !mask_selects(mask, mdt, mmode, r)) return;  // the fix-up writes 0
            T acc = warp_range<SR, T>(b, e, idx, val, x, lane);
            if (lane == 0) chunk_out[k] = acc;
            return;
        }
    }
}

// One thread per split row: fold its chunk partials in order.
template <int SR, typename T>
__global__ void k_spmv_split_fixup(const int32_t* __restrict__ split_rows, const int32_t* __restrict__ split_first,
                                   int64_t nsplit, const T* __restrict__ chunk_out, T* __restrict__ y, int accum,
                                   const void* mask, int mdt, int mmode) {
    using S = Semiring<SR, T>;
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nsplit) return;
    const int32_t r = split_rows[k];
    if (mask && !mask_selects(mask, mdt, mmode, r)) {
        y[r] = T(0);
        return;
    }
    T acc = S::identity();
    for (int32_t c = split_first[k]; c < split_first[k + 1]; c++) acc = S::add(acc, chunk_out[c]);
    y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
}

__global__ void k_bin_keys(const int32_t* ptr, int64_t n, uint32_t* key, int32_t* id) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) {
        key[i] = (uint32_t)bin_of_degree(ptr[i + 1] - ptr[i]);
        id[i] = (int32_t)i;
    }
}

}  // namespace

// Binned layout of one CSR orientation (held by the view's owner).
struct RowBins {
    BinTable bt{};
    int32_t* perm = nullptr;         // rows sorted by bin (stable)
    int32_t* chunk_row = nullptr;    // split chunks: row and first entry
    int32_t* chunk_beg = nullptr;
    int32_t* split_rows = nullptr;   // split rows and their first chunk (nsplit + 1)
    int32_t* split_first = nullptr;
    int64_t nsplit = 0, nchunks = 0;
    void* chunk_out = nullptr;
    int64_t blocks = 0;
};

void free_bins(RowBins* b) {
    if (!b) return;
    cudaFree(b->perm);
    cudaFree(b->chunk_row);
    cudaFree(b->chunk_beg);
    cudaFree(b->split_rows);
    cudaFree(b->split_first);
    cudaFree(b->chunk_out);
    delete b;
}

int build_bins(const CsrView& v, int elem_bytes, RowBins** out, cudaStream_t s) {
    RowBins* rb = new RowBins();
    const int64_t n = v.nrows;
    GBK_CUDA(cudaMalloc(&rb->perm, 4 * (n > 0 ? n : 1)));
    std::vector<int64_t> counts(kNumBins, 0);
    if (n > 0) {
        uint32_t *key = nullptr, *key2 = nullptr;
        int32_t* id = nullptr;
        GBK_CUDA(cudaMalloc(&key, 4 * n));
        GBK_CUDA(cudaMalloc(&key2, 4 * n));
        GBK_CUDA(cudaMalloc(&id, 4 * n));
        k_bin_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v.ptr, n, key, id);
        GBK_LAUNCHED();
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, id, rb->perm, (int)n, 0, 4, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, tb));
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, id, rb->perm, (int)n, 0, 4, s));
        count_launch(1);
        std::vector<uint32_t> hk(n);
        GBK_CUDA(cudaMemcpyAsync(hk.data(), key2, 4 * n, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        for (uint32_t b : hk) counts[b]++;
        cudaFree(tmp);
        cudaFree(key);
        cudaFree(key2);
        cudaFree(id);
    }
    // split rows -> chunk table (host: few rows)
    const int64_t split_begin = n - counts[kBinSplit];
    rb->nsplit = counts[kBinSplit];
    std::vector<int32_t> chunk_row, chunk_beg, split_first;
    if (rb->nsplit > 0) {
        std::vector<int32_t> rows(rb->nsplit), hp(n + 1);
        GBK_CUDA(cudaMemcpyAsync(rows.data(), rb->perm + split_begin, 4 * rb->nsplit, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaMemcpyAsync(hp.data(), v.ptr, 4 * (n + 1), cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        for (int32_t r : rows) {
            split_first.push_back((int32_t)chunk_row.size());
            for (int32_t b = hp[r]; b < hp[r + 1]; b += kSplitNnz) {
                chunk_row.push_back(r);
                chunk_beg.push_back(b);
            }
        }
        split_first.push_back((int32_t)chunk_row.size());
        rb->nchunks = (int64_t)chunk_row.size();
        GBK_CUDA(cudaMalloc(&rb->chunk_row, 4 * rb->nchunks));
        GBK_CUDA(cudaMalloc(&rb->chunk_beg, 4 * rb->nchunks));
        GBK_CUDA(cudaMalloc(&rb->split_rows, 4 * rb->nsplit));
        GBK_CUDA(cudaMalloc(&rb->split_first, 4 * (rb->nsplit + 1)));
        GBK_CUDA(cudaMalloc(&rb->chunk_out, (size_t)elem_bytes * rb->nchunks));
        GBK_CUDA(cudaMemcpyAsync(rb->chunk_row, chunk_row.data(), 4 * rb->nchunks, cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaMemcpyAsync(rb->chunk_beg, chunk_beg.data(), 4 * rb->nchunks, cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaMemcpyAsync(rb->split_rows, rows.data(), 4 * rb->nsplit, cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaMemcpyAsync(rb->split_first, split_first.data(), 4 * (rb->nsplit + 1), cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaStreamSynchronize(s));
    }
    // block table: items in bin order (perm is sorted by bin), CTAs heaviest bin first
    int64_t blk = 0, item = 0;
    const int per_block[kNumBins] = {kBinThreads, kBinThreads, kBinThreads / 2, kBinThreads / 4, kBinThreads / 8,
                                     kBinThreads / 16, kBinThreads / 32, kBinThreads / 32, kBinThreads / 32};
    for (int b = 0; b < kNumBins; b++) {
        rb->bt.item_start[b] = (int32_t)item;
        rb->bt.items[b] = (int32_t)((b == kBinSplit) ? rb->nchunks : counts[b]);
        item += counts[b];
    }
    for (int b = kNumBins - 1; b >= 0; b--) {
        rb->bt.block_start[b] = (int32_t)blk;
        blk += (rb->bt.items[b] + per_block[b] - 1) / per_block[b];
        rb->bt.block_end[b] = (int32_t)blk;
    }
    rb->blocks = blk;
    *out = rb;
    return GBK_SUCCESS;
}

template <int SR, typename T>
int spmv_binned_t(const RowBins* rb, const CsrView& v, int accum, const T* x, T* y, const void* mask, int mdt,
                  int mmode, cudaStream_t s) {
    if (rb->blocks > 0) {
        k_spmv_binned<SR, T><<<(unsigned)rb->blocks, kBinThreads, 0, s>>>(
            rb->bt, v.ptr, v.idx, (const T*)v.val, rb->perm, rb->chunk_row, rb->chunk_beg, x, y, accum, mask, mdt,
            mmode, (T*)rb->chunk_out);
        GBK_LAUNCHED();
    }
    if (rb->nsplit > 0) {
        k_spmv_split_fixup<SR, T><<<(unsigned)((rb->nsplit + 127) / 128), 128, 0, s>>>(
            rb->split_rows, rb->split_first, rb->nsplit, (const T*)rb->chunk_out, y, accum, mask, mdt, mmode);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

template <typename T>
int spmv_binned_dispatch(const RowBins* rb, const CsrView& v, int sr, int accum, const T* x, T* y, const void* mask,
                         int mdt, int mmode, cudaStream_t s) {
    switch (sr) {
        case GBK_PLUS_TIMES: return spmv_binned_t<GBK_PLUS_TIMES, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_LOR_LAND: return spmv_binned_t<GBK_LOR_LAND, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_FIRST_MIN: return spmv_binned_t<GBK_FIRST_MIN, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_PLUS_SECOND: return spmv_binned_t<GBK_PLUS_SECOND, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_STRUCTURAL_BOOL: return spmv_binned_t<GBK_STRUCTURAL_BOOL, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_PLUS: return spmv_binned_t<GBK_MIN_PLUS, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_SECOND: return spmv_binned_t<GBK_MIN_SECOND, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_NOTEQ: return spmv_binned_t<GBK_MIN_NOTEQ, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_PLUS_ONE: return spmv_binned_t<GBK_PLUS_ONE, T>(rb, v, accum, x, y, mask, mdt, mmode, s);
    }
    set_error("binned SpMV: semiring %d not associative", sr);
    return GBK_UNSUPPORTED;
}

int spmv_binned(const RowBins* rb, const CsrView& v, int sr, int accum, int dtype, const void* x, void* y,
                const void* mask, int mdt, int mmode, cudaStream_t s) {
    if (dtype == GBK_F32)
        return spmv_binned_dispatch<float>(rb, v, sr, accum, (const float*)x, (float*)y, mask, mdt, mmode, s);
    return spmv_binned_dispatch<int32_t>(rb, v, sr, accum, (const int32_t*)x, (int32_t*)y, mask, mdt, mmode, s);
}

}  // namespace gbk
