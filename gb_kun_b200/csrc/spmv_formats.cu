// Optimised storage formats: SELL-C-sigma, segmented CSR (CSR_SEG) and LAV.
//
// All three are built on the device from the CSR (and, for A^T, the CSC),
// replacing MatrixSellC::build (src/backend/matrix/containers/sell_c/build.hpp:27-295),
// MatrixSegmentedCSR::build (seg_csr/build.hpp:23-169) and MatrixLAV::build
// (lav/build.hpp:3-212), which build serially on the host.
//
// SELL-C-sigma (C = 32): rows are sorted by degree, descending, inside
// windows of sigma rows; slices of 32 consecutive sorted rows are stored
// column-major and padded to the slice's longest row, so one warp reads one
// slice with fully coalesced 128-byte loads, lane = row.  Slices the
// reference calls problematic (padding >= 2x and > 1024 nonzeros,
// build.hpp:147-155) and slices longer than kSellMaxLen go to an overflow
// CSR handled by the merge-path kernel, so no warp walks a hub row alone.
// (The reference computes problematic chunks and then discards the result,
// spmv_sell_c.h:98-139; here they are computed.)
//
// CSR_SEG and LAV: columns are cut into segments (LAV after renumbering
// columns by descending in-degree and splitting off the 20 % least-used
// columns as one "sparse" segment).  Each (segment, row) pair with entries
// becomes one virtual row of a segment-major CSR; the merge-path kernel
// computes every virtual row, and a merge kernel folds each original row's
// partials in segment order: y = accum(y, add over segments), as the
// reference's scatter-merge does (spmv_seg.h:229-298, spmv_lav.h:124-156).
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace gbk {

constexpr int kSellC = 32;
constexpr int kSellMaxLen = 1 << 30;  // long slices are cut into work items instead
constexpr int kSellChunk = 64;        // slice steps per work item (one warp)
constexpr int kSellUnroll = 8;        // steps per pipelined load group
constexpr int kHotThreads = 1024;     // persistent hot-x CTA: one per SM
#ifndef GBK_SELL_PIECE
#define GBK_SELL_PIECE 256
#endif
constexpr int kSellPiece = GBK_SELL_PIECE;  // rows longer than this are cut into pieces of this many entries
constexpr int kMaxHotBytes = 212992;  // shared memory for staged x (208 KiB)

struct SellC {
    int64_t n = 0;           // rows
    int64_t nslices = 0;
    int32_t sigma = 1;
    int32_t* perm = nullptr;      // sorted position -> row
    int32_t* slice_len = nullptr; // -1 marks an overflow slice
    int64_t* slice_ptr = nullptr; // start of each slice in col / val
    int32_t* col = nullptr;       // column-major padded, -1 = padding
    void* val = nullptr;
    int64_t padded = 0;           // stored entries (including padding)
    // overflow rows (long or problematic slices) as a compact CSR
    int64_t nov = 0;
    int32_t* ov_rows = nullptr;   // original row ids
    CsrView ov;                   // rows 0..nov-1 of the overflow CSR
    void* ov_out = nullptr;       // nov partial results
    // warp work items: kSellChunk steps of one slice each
    int64_t nitems = 0;
    int32_t* item_slice = nullptr;
    int32_t* item_j0 = nullptr;
    int32_t* slice_item0 = nullptr;  // nslices + 1
    void* item_out = nullptr;        // 32 partials per item of a multi-item slice
    int64_t nmulti = 0;
    int32_t* multi = nullptr;        // slices with more than one item
    // hot-x: columns renumbered by in-degree; x[0, hot) staged in shared memory
    int32_t hot = 0;
    int64_t ncols = 0;
    int32_t* new_to_old = nullptr;
    void* xr = nullptr;              // renumbered x (ncols)
    // rows longer than kSellPiece are cut into pieces of kSellPiece entries,
    // stored as extra rows nreal, nreal + 1, ... whose sums go to `piece`;
    // k_piece_fold adds each long row's pieces in order
    int64_t nreal = 0;
    int64_t npieces = 0;
    void* piece = nullptr;
    int64_t nlong = 0;
    int32_t* long_rows = nullptr;
    int32_t* long_p0 = nullptr;      // nlong + 1 offsets into piece
};

struct SegCsr {
    int64_t n = 0;          // rows of the matrix
    int64_t nvrows = 0;     // virtual (segment, row) rows
    int32_t nsegments = 0;
    CsrView v;              // segment-major virtual CSR
    int32_t* merge_ptr = nullptr;  // n + 1, into merge_idx
    int32_t* merge_idx = nullptr;  // virtual rows of each row, in segment order
    void* partial = nullptr;       // nvrows results
    int32_t* col_new_to_old = nullptr;  // LAV only: x reorder
    void* xr = nullptr;                 // LAV only: reordered x (ncols)
    int64_t ncols = 0;
    SegSmem* staged = nullptr;          // LAV only: the renumbered matrix in staged windows
    int64_t dense_cols = 0;             // LAV only: renumbered columns holding the dense fraction of nnz
};

namespace {

inline unsigned blocks_for(int64_t work, int threads = 256) {
    int64_t b = (work + threads - 1) / threads;
    return (unsigned)(b > 0 ? b : 1);
}

// ---------------------------------------------------------------------------
// SELL-C kernels

// Result of stored row r: a real row gets accum(y, acc), a piece of a long
// row (r >= nreal) parks its sum for k_piece_fold.
template <typename T>
__device__ __forceinline__ void sell_store(T* y, T* piece, int64_t nreal, int32_t r, T acc, int accum) {
    if (r < nreal)
        y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
    else
        piece[r - nreal] = acc;
}

// One warp per work item: steps [j0, j0 + kSellChunk) of one slice.  The loop
// is software-pipelined: the col / val group of the next kSellUnroll steps is
// loaded before the x values of the current group are gathered, so two
// dependent memory round trips overlap.  A slice cut into several items
// leaves per-item partials that k_sell_fold combines in item order.
template <int SR, typename T>
__global__ void __launch_bounds__(256) k_sell_items(const int32_t* __restrict__ item_slice,
                                                    const int32_t* __restrict__ item_j0,
                                                    const int32_t* __restrict__ slice_item0,
                                                    const int32_t* __restrict__ slice_len,
                                                    const int64_t* __restrict__ slice_ptr,
                                                    const int32_t* __restrict__ col, const T* __restrict__ val,
                                                    const int32_t* __restrict__ perm, int64_t n, int64_t nitems,
                                                    const T* __restrict__ x, T* __restrict__ y, int accum,
                                                    T* __restrict__ item_out, int64_t nreal, T* __restrict__ piece) {
    using S = Semiring<SR, T>;
    constexpr int U = kSellUnroll;
    const int lane = threadIdx.x & 31;
    const int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (k >= nitems) return;
    const int32_t s = item_slice[k];
    const int32_t j0 = item_j0[k];
    const int32_t j1 = min(j0 + kSellChunk, slice_len[s]);
    const int64_t base = slice_ptr[s] + lane;
    const uint64_t pol = policy_evict_last();
    T acc = S::identity();
    int c[U];
    T a[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const bool in = j0 + u < j1;
        c[u] = in ? ld_stream(col + base + (int64_t)(j0 + u) * kSellC) : -1;
        a[u] = in ? ld_stream(val + base + (int64_t)(j0 + u) * kSellC) : T(0);
    }
    for (int j = j0; j < j1; j += U) {
        int cn[U];
        T an[U];
        const int jn = j + U;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool in = jn + u < j1;
            cn[u] = in ? ld_stream(col + base + (int64_t)(jn + u) * kSellC) : -1;
            an[u] = in ? ld_stream(val + base + (int64_t)(jn + u) * kSellC) : T(0);
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
    if (slice_item0[s + 1] - slice_item0[s] == 1) {
        const int64_t p = (int64_t)s * kSellC + lane;
        if (p < n) sell_store<T>(y, piece, nreal, perm[p], acc, accum);
    } else {
        item_out[k * kSellC + lane] = acc;
    }
}

// Hot-x variant: columns are renumbered by in-degree (descending), so the x
// values of the `hot` most used columns form the prefix x[0, hot).  Each
// persistent CTA copies that prefix into shared memory once, and gathers of
// hot columns read shared memory instead of making an L2 round trip.
template <int SR, typename T>
__global__ void __launch_bounds__(kHotThreads) k_sell_items_hot(
    const int32_t* __restrict__ item_slice, const int32_t* __restrict__ item_j0,
    const int32_t* __restrict__ slice_item0, const int32_t* __restrict__ slice_len,
    const int64_t* __restrict__ slice_ptr, const int32_t* __restrict__ col, const T* __restrict__ val,
    const int32_t* __restrict__ perm, int64_t n, int64_t nitems, int hot, const T* __restrict__ x,
    T* __restrict__ y, int accum, T* __restrict__ item_out, int64_t nreal, T* __restrict__ piece) {
    using S = Semiring<SR, T>;
    constexpr int U = kSellUnroll;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sx = reinterpret_cast<T*>(smem_raw);
    for (int i = threadIdx.x; i < hot; i += kHotThreads) sx[i] = x[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (kHotThreads / 32);
    const uint64_t pol = policy_evict_last();
    for (int64_t k = (int64_t)blockIdx.x * (kHotThreads / 32) + (threadIdx.x >> 5); k < nitems; k += warps) {
        const int32_t s = item_slice[k];
        const int32_t j0 = item_j0[k];
        const int32_t j1 = min(j0 + kSellChunk, slice_len[s]);
        const int64_t base = slice_ptr[s] + lane;
        T acc = S::identity();
        int c[U];
        T a[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool in = j0 + u < j1;
            c[u] = in ? ld_stream(col + base + (int64_t)(j0 + u) * kSellC) : -1;
            a[u] = in ? ld_stream(val + base + (int64_t)(j0 + u) * kSellC) : T(0);
        }
        for (int j = j0; j < j1; j += U) {
            int cn[U];
            T an[U];
            const int jn = j + U;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool in = jn + u < j1;
                cn[u] = in ? ld_stream(col + base + (int64_t)(jn + u) * kSellC) : -1;
                an[u] = in ? ld_stream(val + base + (int64_t)(jn + u) * kSellC) : T(0);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (c[u] >= 0) {
                    const T xv = c[u] < hot ? sx[c[u]] : ld_keep(x + c[u], pol);
                    acc = S::add(acc, S::mul(a[u], xv));
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                c[u] = cn[u];
                a[u] = an[u];
            }
        }
        if (slice_item0[s + 1] - slice_item0[s] == 1) {
            const int64_t p = (int64_t)s * kSellC + lane;
            if (p < n) sell_store<T>(y, piece, nreal, perm[p], acc, accum);
        } else {
            item_out[k * kSellC + lane] = acc;
        }
    }
}

// x in the renumbered column order: xr[i] = x[new_to_old[i]]
template <typename T>
__global__ void k_permute_x(const T* __restrict__ x, const int32_t* __restrict__ new_to_old, int64_t n,
                            T* __restrict__ xr) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) xr[i] = x[new_to_old[i]];
}

// stored column ids -> renumbered ids (padding -1 stays)
__global__ void k_renumber(int32_t* col, int64_t m, const int32_t* __restrict__ old_to_new) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < m && col[e] >= 0) col[e] = old_to_new[col[e]];
}

// Slices cut into several items: fold the partials of each lane in item order.
template <int SR, typename T>
__global__ void k_sell_fold(const int32_t* __restrict__ multi, int64_t nmulti, const int32_t* __restrict__ slice_item0,
                            const T* __restrict__ item_out, const int32_t* __restrict__ perm, int64_t n,
                            T* __restrict__ y, int accum, int64_t nreal, T* __restrict__ piece) {
    using S = Semiring<SR, T>;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nmulti * kSellC) return;
    const int32_t s = multi[t / kSellC];
    const int lane = (int)(t % kSellC);
    T acc = S::identity();
    for (int32_t k = slice_item0[s]; k < slice_item0[s + 1]; k++) acc = S::add(acc, item_out[(int64_t)k * kSellC + lane]);
    const int64_t p = (int64_t)s * kSellC + lane;
    if (p < n) sell_store<T>(y, piece, nreal, perm[p], acc, accum);
}

// Work items of a slice: ceil(len / kSellChunk), at least 1 (empty slices
// still write their rows); overflow slices have none.
__global__ void k_sell_item_counts(const int32_t* len, int64_t ns, int32_t* cnt) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s < ns) cnt[s] = len[s] < 0 ? 0 : max(1, (len[s] + kSellChunk - 1) / kSellChunk);
    if (s == ns) cnt[s] = 0;
}

__global__ void k_sell_item_fill(const int32_t* cnt, const int32_t* first, int64_t ns, int32_t* item_slice,
                                 int32_t* item_j0, int32_t* multi_flag) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= ns) return;
    for (int32_t c = 0; c < cnt[s]; c++) {
        item_slice[first[s] + c] = (int32_t)s;
        item_j0[first[s] + c] = c * kSellChunk;
    }
    multi_flag[s] = cnt[s] > 1 ? 1 : 0;
}

__global__ void k_compact_flags(const int32_t* flag, const int32_t* pos, int64_t n, int32_t* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n && flag[i]) out[pos[i]] = (int32_t)i;
}

template <typename T>
__global__ void k_scatter_rows(const int32_t* __restrict__ rows, const T* __restrict__ part, int64_t nr,
                               T* __restrict__ y, int accum, int64_t nreal, T* __restrict__ piece) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nr) return;
    sell_store<T>(y, piece, nreal, rows[k], part[k], accum);
}

// Each long row: its pieces' sums added in piece order, then the accumulator.
template <int SR, typename T>
__global__ void k_piece_fold(const int32_t* __restrict__ long_rows, const int32_t* __restrict__ long_p0,
                             int64_t nlong, const T* __restrict__ piece, T* __restrict__ y, int accum) {
    using S = Semiring<SR, T>;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nlong) return;
    T acc = S::identity();
    for (int32_t k = long_p0[j]; k < long_p0[j + 1]; ++k) acc = S::add(acc, piece[k]);
    const int32_t r = long_rows[j];
    y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
}

// Virtual rows of the SELL-C build: real rows of at most L entries keep
// their id; longer rows are replaced by pieces of L entries with ids
// n + pstart[r] + j.  vlen < 0 marks a replaced real row.
__global__ void k_piece_counts(const int32_t* __restrict__ ptr, int64_t n, int L, int32_t* np) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < n) {
        const int32_t d = ptr[r + 1] - ptr[r];
        np[r] = d > L ? (d + L - 1) / L : 0;
    } else if (r == n) {
        np[n] = 0;
    }
}

__global__ void k_virtual_rows(const int32_t* __restrict__ ptr, int64_t n, int L, const int32_t* __restrict__ pstart,
                               int32_t* vstart, int32_t* vlen, int32_t* keep) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int32_t b = ptr[r], d = ptr[r + 1] - ptr[r];
    if (d <= L) {
        vstart[r] = b;
        vlen[r] = d;
        keep[r] = 1;
        return;
    }
    vlen[r] = -1;
    keep[r] = 0;
    const int32_t np = (d + L - 1) / L;
    for (int32_t j = 0; j < np; ++j) {
        const int64_t id = n + pstart[r] + j;
        vstart[id] = b + j * L;
        vlen[id] = min(L, d - j * L);
        keep[id] = 1;
    }
}

__global__ void k_vsigma_keys(const int32_t* __restrict__ vlen, const int32_t* __restrict__ idl, int64_t nv,
                              int32_t sigma, unsigned long long* keys, int32_t* vals) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const unsigned long long win = (unsigned long long)(i / sigma);
    keys[i] = (win << 32) | (unsigned long long)(uint32_t)(0x7fffffff - vlen[idl[i]]);
    vals[i] = idl[i];
}

__global__ void k_long_flags(const int32_t* __restrict__ np, int64_t n, int32_t* flag) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < n) flag[r] = np[r] > 0;
    else if (r == n) flag[n] = 0;
}

__global__ void k_long_list(const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                            const int32_t* __restrict__ pstart, int64_t n, int64_t npieces, int32_t* rows,
                            int32_t* p0) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < n && flag[r]) {
        rows[pos[r]] = (int32_t)r;
        p0[pos[r]] = pstart[r];
    }
    if (r == n) p0[pos[n]] = (int32_t)npieces;
}

// SELL-C build helpers


// one warp per slice: longest row and nonzero count; classify overflow
__global__ void k_slice_stats(const int32_t* deg, const int32_t* perm, int64_t n, int64_t nslices, int32_t* len,
                              int64_t* stored, int32_t* is_ov) {
    const int lane = threadIdx.x & 31;
    const int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (s >= nslices) return;
    const int64_t p = s * kSellC + lane;
    int d = (p < n) ? deg[perm[p]] : 0;
    int mx = d;
    long long sum = d;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        sum += __shfl_xor_sync(0xffffffffu, sum, off);
    }
    if (lane == 0) {
        const bool problematic = ((long long)mx * kSellC >= 2 * sum) && (sum > 1024);
        const bool ov = problematic || mx > kSellMaxLen;
        len[s] = ov ? -1 : mx;
        stored[s] = ov ? 0 : (int64_t)mx * kSellC;
        is_ov[s] = ov ? 1 : 0;
    }
}

template <typename T>
__global__ void k_sell_fill(const int32_t* __restrict__ vstart, const int32_t* __restrict__ vlen,
                            const int32_t* __restrict__ idx, const T* __restrict__ val,
                            const int32_t* __restrict__ perm, const int32_t* __restrict__ len,
                            const int64_t* __restrict__ sptr, int64_t n, int32_t* __restrict__ col,
                            T* __restrict__ sval) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int64_t s = p / kSellC;
    if (len[s] < 0) return;
    const int lane = (int)(p % kSellC);
    const int32_t r = perm[p];
    const int64_t base = sptr[s] + lane;
    for (int32_t e = vstart[r], j = 0; j < vlen[r]; e++, j++) {
        col[base + (int64_t)j * kSellC] = idx[e];
        sval[base + (int64_t)j * kSellC] = val[e];
    }
}

// rows of overflow slices, in sorted order
__global__ void k_ov_flags(const int32_t* is_ov, const int32_t* perm, int64_t n, int32_t* flag) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < n) flag[p] = is_ov[p / kSellC];
}

__global__ void k_ov_compact(const int32_t* flag, const int32_t* pos, const int32_t* perm, const int32_t* deg,
                             int64_t n, int32_t* rows, int32_t* rdeg) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < n && flag[p]) {
        rows[pos[p]] = perm[p];
        rdeg[pos[p]] = deg[perm[p]];
    }
}

// copy listed rows of a CSR into a compact CSR (warp per row)
template <typename T>
__global__ void k_gather_rows(const int32_t* __restrict__ vstart, const int32_t* __restrict__ vlen,
                              const int32_t* __restrict__ idx, const T* __restrict__ val,
                              const int32_t* __restrict__ rows, const int32_t* __restrict__ optr, int64_t nr,
                              int32_t* __restrict__ oidx, T* __restrict__ oval) {
    const int lane = threadIdx.x & 31;
    const int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (k >= nr) return;
    const int32_t r = rows[k];
    const int32_t b = vstart[r], e = vstart[r] + vlen[r], o = optr[k];
    for (int32_t q = b + lane; q < e; q += 32) {
        oidx[o + (q - b)] = idx[q];
        oval[o + (q - b)] = val[q];
    }
}

// ---------------------------------------------------------------------------
// segmented (CSR_SEG / LAV) kernels

template <int SR, typename T>
__global__ void k_seg_merge(const int32_t* __restrict__ mptr, const int32_t* __restrict__ midx,
                            const T* __restrict__ part, int64_t n, T* __restrict__ y, int accum) {
    using S = Semiring<SR, T>;
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    T acc = S::identity();
    for (int32_t k = mptr[r]; k < mptr[r + 1]; k++) acc = S::add(acc, part[midx[k]]);
    y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
}

template <typename T>
__global__ void k_reorder_x(const T* __restrict__ x, const int32_t* __restrict__ new_to_old, int64_t n,
                            T* __restrict__ xr) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) xr[i] = x[new_to_old[i]];
}

// LAV column renumbering on the device (lav/build.hpp:113-141): in-degree of
// every column, columns sorted by it (descending, ties in column order: a
// stable radix sort), the inverse map, and the stored column ids relabelled.
// (k_col_hist and k_invert_perm, shared with the SELL-C renumbering, are
// defined with the SELL-C build below.)
__global__ void k_col_hist(const int32_t* __restrict__ idx, int64_t nnz, int32_t* __restrict__ cdeg);
__global__ void k_invert_perm(const int32_t* new_to_old, int64_t n, int32_t* old_to_new);

__global__ void k_iota32(int32_t* __restrict__ v, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

__global__ void k_relabel(const int32_t* __restrict__ idx, int64_t nnz, const int32_t* __restrict__ old_to_new,
                          int32_t* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = old_to_new[idx[e]];
}

// First renumbered column at which the running in-degree sum reaches
// `target` (the reference's dense_threshold); one thread, binary search over
// the inclusive scan of the sorted degrees.
__global__ void k_dense_threshold(const long long* __restrict__ acc, int64_t n, long long target,
                                  long long* __restrict__ out) {
    int64_t lo = 0, hi = n;  // first c with acc[c] >= target, n if none
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (acc[mid] >= target)
            hi = mid;
        else
            lo = mid + 1;
    }
    *out = lo;
}

// Segment id of every entry: key = (segment << 32) | row, value = entry position.
__global__ void k_seg_keys(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, int64_t nrows,
                           int64_t nnz, const int32_t* __restrict__ col_seg, unsigned long long* __restrict__ keys,
                           int32_t* __restrict__ pos) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int64_t lo = 0, hi = nrows;
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (ptr[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    keys[e] = ((unsigned long long)(uint32_t)col_seg[idx[e]] << 32) | (uint32_t)lo;
    pos[e] = (int32_t)e;
}

// virtual-row boundaries: a new virtual row starts where the (segment, row) key changes
__global__ void k_vrow_flags(const unsigned long long* keys, int64_t nnz, int32_t* flag) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < nnz) flag[e] = (e == 0 || keys[e] != keys[e - 1]) ? 1 : 0;
}

template <typename T>
__global__ void k_vrow_build(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ pos,
                             const int32_t* __restrict__ flag, const int32_t* __restrict__ vid,
                             const int32_t* __restrict__ idx, const T* __restrict__ val,
                             const int32_t* __restrict__ col_map, int64_t nnz, int32_t* __restrict__ vptr,
                             int32_t* __restrict__ vrow, int32_t* __restrict__ oidx, T* __restrict__ oval,
                             int32_t* __restrict__ rowcount) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const int32_t src = pos[e];
    const int32_t c = idx[src];
    oidx[e] = col_map ? col_map[c] : c;
    oval[e] = val[src];
    if (flag[e]) {
        const int32_t v = vid[e];  // exclusive scan of flags
        vptr[v] = (int32_t)e;
        const int32_t r = (int32_t)(keys[e] & 0xffffffffULL);
        vrow[v] = r;
        atomicAdd(&rowcount[r], 1);
    }
}

// merge lists: virtual rows of each original row in segment order.  Virtual
// rows are segment-major, so visiting them in order and appending per row
// keeps segment order; a per-row cursor does the appending.
__global__ void k_merge_fill(const int32_t* __restrict__ vrow, int64_t nv, const int32_t* __restrict__ mptr,
                             int32_t* __restrict__ cursor, int32_t* __restrict__ midx) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const int32_t r = vrow[v];
    const int32_t slot = atomicAdd(&cursor[r], 1);
    midx[mptr[r] + slot] = (int32_t)v;
}

// restore segment order inside each row's merge list (short lists: insertion sort)
__global__ void k_merge_sort(const int32_t* __restrict__ mptr, int64_t n, int32_t* __restrict__ midx) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int32_t b = mptr[r], e = mptr[r + 1];
    for (int32_t i = b + 1; i < e; i++) {
        int32_t v = midx[i];
        int32_t j = i - 1;
        while (j >= b && midx[j] > v) {
            midx[j + 1] = midx[j];
            j--;
        }
        midx[j + 1] = v;
    }
}

int cub_scan_excl(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s) {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&tmp, tb, s));
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int)n, s));
    count_launch(1);
    cudaFreeAsync(tmp, s);
    return GBK_SUCCESS;
}

int free_sell(SellC* f) {
    if (!f) return 0;
    cudaFree(f->perm);
    cudaFree(f->slice_len);
    cudaFree(f->slice_ptr);
    cudaFree(f->col);
    cudaFree(f->val);
    cudaFree(f->ov_rows);
    cudaFree(f->ov_out);
    cudaFree(f->item_slice);
    cudaFree(f->item_j0);
    cudaFree(f->slice_item0);
    cudaFree(f->item_out);
    cudaFree(f->multi);
    cudaFree(f->new_to_old);
    cudaFree(f->xr);
    cudaFree(f->piece);
    cudaFree(f->long_rows);
    cudaFree(f->long_p0);
    free_view(f->ov);
    delete f;
    return 0;
}

int free_seg(SegCsr* f) {
    if (!f) return 0;
    free_view(f->v);
    cudaFree(f->merge_ptr);
    cudaFree(f->merge_idx);
    cudaFree(f->partial);
    cudaFree(f->col_new_to_old);
    cudaFree(f->xr);
    free_segsmem(f->staged);
    delete f;
    return 0;
}

// ---------------------------------------------------------------------------
// SELL-C build

__global__ void k_col_hist(const int32_t* __restrict__ idx, int64_t nnz, int32_t* __restrict__ cdeg) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < nnz) atomicAdd(&cdeg[idx[e]], 1);
}

__global__ void k_hot_keys(const int32_t* cdeg, int64_t nc, uint32_t* key, int32_t* id) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c < nc) {
        key[c] = (uint32_t)(0x7fffffff - cdeg[c]);
        id[c] = (int32_t)c;
    }
}

__global__ void k_invert_perm(const int32_t* new_to_old, int64_t n, int32_t* old_to_new) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) old_to_new[new_to_old[i]] = (int32_t)i;
}

// Renumber columns by in-degree (descending, stable), as MatrixLAV does
// (src/backend/matrix/containers/lav/build.hpp:113-141), and rewrite the
// stored column ids, so the most used x values form the prefix x[0, hot).
int renumber_hot(const CsrView& a, int32_t hot, SellC* f, cudaStream_t s) {
    const int64_t nc = a.ncols;
    int32_t *cdeg = nullptr, *id = nullptr, *old_to_new = nullptr;
    uint32_t *key = nullptr, *key2 = nullptr;
    GBK_CUDA(cudaMalloc(&cdeg, 4 * nc));
    GBK_CUDA(cudaMalloc(&id, 4 * nc));
    GBK_CUDA(cudaMalloc(&key, 4 * nc));
    GBK_CUDA(cudaMalloc(&key2, 4 * nc));
    GBK_CUDA(cudaMalloc(&old_to_new, 4 * nc));
    GBK_CUDA(cudaMalloc(&f->new_to_old, 4 * nc));
    GBK_CUDA(cudaMemsetAsync(cdeg, 0, 4 * nc, s));
    if (a.nnz > 0) {
        k_col_hist<<<blocks_for(a.nnz), 256, 0, s>>>(a.idx, a.nnz, cdeg);
        GBK_LAUNCHED();
    }
    k_hot_keys<<<blocks_for(nc), 256, 0, s>>>(cdeg, nc, key, id);
    GBK_LAUNCHED();
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, id, f->new_to_old, (int)nc, 0, 32, s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMalloc(&tmp, tb));
    GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, id, f->new_to_old, (int)nc, 0, 32, s));
    count_launch(1);
    k_invert_perm<<<blocks_for(nc), 256, 0, s>>>(f->new_to_old, nc, old_to_new);
    GBK_LAUNCHED();
    if (f->padded > 0) {
        k_renumber<<<blocks_for(f->padded), 256, 0, s>>>(f->col, f->padded, old_to_new);
        GBK_LAUNCHED();
    }
    if (f->ov.nnz > 0) {
        k_renumber<<<blocks_for(f->ov.nnz), 256, 0, s>>>(f->ov.idx, f->ov.nnz, old_to_new);
        GBK_LAUNCHED();
    }
    GBK_CUDA(cudaMalloc(&f->xr, 4 * nc));  // 4-byte element types
    f->hot = (int32_t)(hot < nc ? hot : nc);
    GBK_CUDA(cudaStreamSynchronize(s));
    cudaFree(tmp);
    cudaFree(cdeg);
    cudaFree(id);
    cudaFree(key);
    cudaFree(key2);
    cudaFree(old_to_new);
    return GBK_SUCCESS;
}

template <typename T>
int build_sell(const CsrView& a, int32_t sigma, int32_t hot, int32_t reorder, SellC** out, cudaStream_t s) {
    SellC* f = new SellC();
    f->sigma = sigma;
    f->ncols = a.ncols;
    const int64_t nr = a.nrows;
    f->nreal = nr;
    // virtual rows: rows of at most kSellPiece entries, and kSellPiece-entry
    // pieces of the longer ones (ids nr, nr + 1, ...)
    int32_t *np = nullptr, *pstart = nullptr;
    GBK_CUDA(cudaMalloc(&np, sizeof(int32_t) * (nr + 1)));
    GBK_CUDA(cudaMalloc(&pstart, sizeof(int32_t) * (nr + 1)));
    k_piece_counts<<<blocks_for(nr + 1), 256, 0, s>>>(a.ptr, nr, kSellPiece, np);
    GBK_LAUNCHED();
    int rc0 = cub_scan_excl(np, pstart, nr + 1, s);
    if (rc0) return rc0;
    int32_t npieces = 0;
    GBK_CUDA(cudaMemcpyAsync(&npieces, pstart + nr, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    f->npieces = npieces;
    const int64_t nvt = nr + npieces;
    int32_t *vstart = nullptr, *deg = nullptr, *keep = nullptr, *kpos = nullptr, *idl = nullptr;
    GBK_CUDA(cudaMalloc(&vstart, sizeof(int32_t) * (nvt > 0 ? nvt : 1)));
    GBK_CUDA(cudaMalloc(&deg, sizeof(int32_t) * (nvt > 0 ? nvt : 1)));  // vlen, indexed by virtual id
    GBK_CUDA(cudaMalloc(&keep, sizeof(int32_t) * (nvt + 1)));
    GBK_CUDA(cudaMalloc(&kpos, sizeof(int32_t) * (nvt + 1)));
    GBK_CUDA(cudaMemsetAsync(keep + nvt, 0, sizeof(int32_t), s));
    if (nr > 0) {
        k_virtual_rows<<<blocks_for(nr), 256, 0, s>>>(a.ptr, nr, kSellPiece, pstart, vstart, deg, keep);
        GBK_LAUNCHED();
    }
    rc0 = cub_scan_excl(keep, kpos, nvt + 1, s);
    if (rc0) return rc0;
    int32_t nv32 = 0;
    GBK_CUDA(cudaMemcpyAsync(&nv32, kpos + nvt, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    const int64_t n = nv32;
    f->n = n;
    f->nslices = (n + kSellC - 1) / kSellC;
    GBK_CUDA(cudaMalloc(&idl, sizeof(int32_t) * (n > 0 ? n : 1)));
    if (nvt > 0) {
        k_compact_flags<<<blocks_for(nvt), 256, 0, s>>>(keep, kpos, nvt, idl);
        GBK_LAUNCHED();
    }
    GBK_CUDA(cudaMalloc(&f->perm, sizeof(int32_t) * (n > 0 ? n : 1)));
    if (sigma > 1 && n > 1) {
        unsigned long long *keys = nullptr, *keys2 = nullptr;
        int32_t* ids = nullptr;
        GBK_CUDA(cudaMalloc(&keys, sizeof(unsigned long long) * n));
        GBK_CUDA(cudaMalloc(&keys2, sizeof(unsigned long long) * n));
        GBK_CUDA(cudaMalloc(&ids, sizeof(int32_t) * n));
        k_vsigma_keys<<<blocks_for(n), 256, 0, s>>>(deg, idl, n, sigma, keys, ids);
        GBK_LAUNCHED();
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, ids, f->perm, (int)n, 0, 64, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, tb));
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, ids, f->perm, (int)n, 0, 64, s));
        count_launch(1);
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(tmp);
        cudaFree(keys);
        cudaFree(keys2);
        cudaFree(ids);
    } else if (n > 0) {
        GBK_CUDA(cudaMemcpyAsync(f->perm, idl, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    // long rows and their piece ranges, for k_piece_fold
    if (npieces > 0) {
        int32_t *lflag = nullptr, *lpos = nullptr;
        GBK_CUDA(cudaMalloc(&lflag, sizeof(int32_t) * (nr + 1)));
        GBK_CUDA(cudaMalloc(&lpos, sizeof(int32_t) * (nr + 1)));
        k_long_flags<<<blocks_for(nr + 1), 256, 0, s>>>(np, nr, lflag);
        GBK_LAUNCHED();
        rc0 = cub_scan_excl(lflag, lpos, nr + 1, s);
        if (rc0) return rc0;
        int32_t nl = 0;
        GBK_CUDA(cudaMemcpyAsync(&nl, lpos + nr, 4, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        f->nlong = nl;
        GBK_CUDA(cudaMalloc(&f->long_rows, sizeof(int32_t) * (nl > 0 ? nl : 1)));
        GBK_CUDA(cudaMalloc(&f->long_p0, sizeof(int32_t) * (nl + 1)));
        k_long_list<<<blocks_for(nr + 1), 256, 0, s>>>(lflag, lpos, pstart, nr, npieces, f->long_rows, f->long_p0);
        GBK_LAUNCHED();
        GBK_CUDA(cudaMalloc(&f->piece, sizeof(T) * npieces));
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(lflag);
        cudaFree(lpos);
    }
    const int64_t ns = f->nslices;
    int32_t* is_ov = nullptr;
    int64_t* stored = nullptr;
    GBK_CUDA(cudaMalloc(&f->slice_len, sizeof(int32_t) * (ns > 0 ? ns : 1)));
    GBK_CUDA(cudaMalloc(&f->slice_ptr, sizeof(int64_t) * (ns + 1)));
    GBK_CUDA(cudaMalloc(&is_ov, sizeof(int32_t) * (ns > 0 ? ns : 1)));
    GBK_CUDA(cudaMalloc(&stored, sizeof(int64_t) * (ns + 1)));
    GBK_CUDA(cudaMemsetAsync(stored, 0, sizeof(int64_t) * (ns + 1), s));
    if (ns > 0) {
        k_slice_stats<<<blocks_for(ns * 32), 256, 0, s>>>(deg, f->perm, n, ns, f->slice_len, stored, is_ov);
        GBK_LAUNCHED();
    }
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, stored, f->slice_ptr, (int)(ns + 1), s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, tb));
        GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, stored, f->slice_ptr, (int)(ns + 1), s));
        count_launch(1);
        GBK_CUDA(cudaMemcpyAsync(&f->padded, f->slice_ptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(tmp);
    }
    GBK_CUDA(cudaMalloc(&f->col, sizeof(int32_t) * (f->padded > 0 ? f->padded : 1)));
    GBK_CUDA(cudaMalloc(&f->val, sizeof(T) * (f->padded > 0 ? f->padded : 1)));
    GBK_CUDA(cudaMemsetAsync(f->col, 0xff, sizeof(int32_t) * (f->padded > 0 ? f->padded : 1), s));
    GBK_CUDA(cudaMemsetAsync(f->val, 0, sizeof(T) * (f->padded > 0 ? f->padded : 1), s));
    if (n > 0) {
        k_sell_fill<T><<<blocks_for(n), 256, 0, s>>>(vstart, deg, a.idx, (const T*)a.val, f->perm, f->slice_len,
                                                      f->slice_ptr, n, f->col, (T*)f->val);
        GBK_LAUNCHED();
    }
    // warp work items
    if (ns > 0) {
        int32_t *cnt = nullptr, *mflag = nullptr, *mpos = nullptr;
        GBK_CUDA(cudaMalloc(&cnt, 4 * (ns + 1)));
        GBK_CUDA(cudaMalloc(&mflag, 4 * (ns + 1)));
        GBK_CUDA(cudaMalloc(&mpos, 4 * (ns + 1)));
        GBK_CUDA(cudaMalloc(&f->slice_item0, 4 * (ns + 1)));
        k_sell_item_counts<<<blocks_for(ns + 1), 256, 0, s>>>(f->slice_len, ns, cnt);
        GBK_LAUNCHED();
        int rc = cub_scan_excl(cnt, f->slice_item0, ns + 1, s);
        if (rc) return rc;
        int32_t ni = 0;
        GBK_CUDA(cudaMemcpyAsync(&ni, f->slice_item0 + ns, 4, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        f->nitems = ni;
        GBK_CUDA(cudaMalloc(&f->item_slice, 4 * (ni > 0 ? ni : 1)));
        GBK_CUDA(cudaMalloc(&f->item_j0, 4 * (ni > 0 ? ni : 1)));
        GBK_CUDA(cudaMalloc(&f->item_out, sizeof(T) * kSellC * (ni > 0 ? ni : 1)));
        GBK_CUDA(cudaMemsetAsync(mflag + ns, 0, 4, s));
        k_sell_item_fill<<<blocks_for(ns), 256, 0, s>>>(cnt, f->slice_item0, ns, f->item_slice, f->item_j0, mflag);
        GBK_LAUNCHED();
        rc = cub_scan_excl(mflag, mpos, ns + 1, s);
        if (rc) return rc;
        int32_t nm = 0;
        GBK_CUDA(cudaMemcpyAsync(&nm, mpos + ns, 4, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        f->nmulti = nm;
        GBK_CUDA(cudaMalloc(&f->multi, 4 * (nm > 0 ? nm : 1)));
        if (nm > 0) {
            k_compact_flags<<<blocks_for(ns), 256, 0, s>>>(mflag, mpos, ns, f->multi);
            GBK_LAUNCHED();
        }
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(cnt);
        cudaFree(mflag);
        cudaFree(mpos);
    }
    // overflow rows
    if (n > 0) {
        int32_t *flag = nullptr, *pos = nullptr, *rdeg = nullptr;
        GBK_CUDA(cudaMalloc(&flag, sizeof(int32_t) * (n + 1)));
        GBK_CUDA(cudaMalloc(&pos, sizeof(int32_t) * (n + 1)));
        GBK_CUDA(cudaMemsetAsync(flag + n, 0, sizeof(int32_t), s));
        k_ov_flags<<<blocks_for(n), 256, 0, s>>>(is_ov, f->perm, n, flag);
        GBK_LAUNCHED();
        int rc = cub_scan_excl(flag, pos, n + 1, s);
        if (rc) return rc;
        int32_t nov = 0;
        GBK_CUDA(cudaMemcpyAsync(&nov, pos + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        f->nov = nov;
        if (nov > 0) {
            GBK_CUDA(cudaMalloc(&f->ov_rows, sizeof(int32_t) * nov));
            GBK_CUDA(cudaMalloc(&rdeg, sizeof(int32_t) * (nov + 1)));
            GBK_CUDA(cudaMemsetAsync(rdeg + nov, 0, sizeof(int32_t), s));
            k_ov_compact<<<blocks_for(n), 256, 0, s>>>(flag, pos, f->perm, deg, n, f->ov_rows, rdeg);
            GBK_LAUNCHED();
            CsrView& o = f->ov;
            o.nrows = nov;
            o.ncols = a.ncols;
            GBK_CUDA(cudaMalloc(&o.ptr, sizeof(int32_t) * (nov + 1)));
            rc = cub_scan_excl(rdeg, o.ptr, nov + 1, s);
            if (rc) return rc;
            int32_t onnz = 0;
            GBK_CUDA(cudaMemcpyAsync(&onnz, o.ptr + nov, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            GBK_CUDA(cudaStreamSynchronize(s));
            o.nnz = onnz;
            GBK_CUDA(cudaMalloc(&o.idx, sizeof(int32_t) * (onnz > 0 ? onnz : 1)));
            GBK_CUDA(cudaMalloc(&o.val, sizeof(T) * (onnz > 0 ? onnz : 1)));
            k_gather_rows<T><<<blocks_for(nov * 32), 256, 0, s>>>(vstart, deg, a.idx, (const T*)a.val, f->ov_rows,
                                                                   o.ptr, nov, o.idx, (T*)o.val);
            GBK_LAUNCHED();
            rc = build_tiles(o, sizeof(T), s);
            if (rc) return rc;
            GBK_CUDA(cudaMalloc(&f->ov_out, sizeof(T) * nov));
        }
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(flag);
        cudaFree(pos);
        cudaFree(rdeg);
    }
    cudaFree(is_ov);
    cudaFree(stored);
    cudaFree(deg);
    cudaFree(vstart);
    cudaFree(np);
    cudaFree(pstart);
    cudaFree(keep);
    cudaFree(kpos);
    cudaFree(idl);
    if ((hot > 0 || reorder) && a.ncols > 0) {
        int rc = renumber_hot(a, hot, f, s);
        if (rc) return rc;
    }
    *out = f;
    return GBK_SUCCESS;
}

// ---------------------------------------------------------------------------
// CSR_SEG / LAV build: col_seg[c] = segment of column c, col_map = optional
// column renumbering applied to the stored column ids (LAV).

template <typename T>
int build_segmented(const CsrView& a, const std::vector<int32_t>& col_seg_h, const int32_t* col_map_d,
                    int32_t nseg, SegCsr* f, cudaStream_t s) {
    const int64_t n = a.nrows, nnz = a.nnz;
    f->n = n;
    f->ncols = a.ncols;
    f->nsegments = nseg;
    int32_t* col_seg = nullptr;
    GBK_CUDA(cudaMalloc(&col_seg, sizeof(int32_t) * (a.ncols > 0 ? a.ncols : 1)));
    GBK_CUDA(cudaMemcpyAsync(col_seg, col_seg_h.data(), sizeof(int32_t) * a.ncols, cudaMemcpyHostToDevice, s));
    CsrView& v = f->v;
    v.ncols = a.ncols;
    v.nnz = nnz;
    GBK_CUDA(cudaMalloc(&f->merge_ptr, sizeof(int32_t) * (n + 1)));
    GBK_CUDA(cudaMemsetAsync(f->merge_ptr, 0, sizeof(int32_t) * (n + 1), s));
    GBK_CUDA(cudaMalloc(&v.idx, sizeof(int32_t) * (nnz > 0 ? nnz : 1)));
    GBK_CUDA(cudaMalloc(&v.val, sizeof(T) * (nnz > 0 ? nnz : 1)));
    if (nnz > 0) {
        unsigned long long *keys = nullptr, *keys2 = nullptr;
        int32_t *pos = nullptr, *pos2 = nullptr, *flag = nullptr, *vid = nullptr;
        GBK_CUDA(cudaMalloc(&keys, 8 * nnz));
        GBK_CUDA(cudaMalloc(&keys2, 8 * nnz));
        GBK_CUDA(cudaMalloc(&pos, 4 * nnz));
        GBK_CUDA(cudaMalloc(&pos2, 4 * nnz));
        GBK_CUDA(cudaMalloc(&flag, 4 * (nnz + 1)));
        GBK_CUDA(cudaMalloc(&vid, 4 * (nnz + 1)));
        k_seg_keys<<<blocks_for(nnz), 256, 0, s>>>(a.ptr, a.idx, n, nnz, col_seg, keys, pos);
        GBK_LAUNCHED();
        // entries in row order: a stable sort on the segment bits suffices
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, pos, pos2, (int)nnz, 32, 64, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, tb));
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, pos, pos2, (int)nnz, 32, 64, s));
        count_launch(1);
        GBK_CUDA(cudaMemsetAsync(flag + nnz, 0, 4, s));
        k_vrow_flags<<<blocks_for(nnz), 256, 0, s>>>(keys2, nnz, flag);
        GBK_LAUNCHED();
        int rc = cub_scan_excl(flag, vid, nnz + 1, s);
        if (rc) return rc;
        int32_t nv = 0;
        GBK_CUDA(cudaMemcpyAsync(&nv, vid + nnz, 4, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        f->nvrows = nv;
        v.nrows = nv;
        int32_t *vrow = nullptr, *rowcount = nullptr;
        GBK_CUDA(cudaMalloc(&v.ptr, 4 * (nv + 1)));
        GBK_CUDA(cudaMalloc(&vrow, 4 * (nv > 0 ? nv : 1)));
        GBK_CUDA(cudaMalloc(&rowcount, 4 * (n + 1)));
        GBK_CUDA(cudaMemsetAsync(rowcount, 0, 4 * (n + 1), s));
        int32_t nnz32 = (int32_t)nnz;
        GBK_CUDA(cudaMemcpyAsync(v.ptr + nv, &nnz32, 4, cudaMemcpyHostToDevice, s));
        k_vrow_build<T><<<blocks_for(nnz), 256, 0, s>>>(keys2, pos2, flag, vid, a.idx, (const T*)a.val, col_map_d,
                                                         nnz, v.ptr, vrow, v.idx, (T*)v.val, rowcount);
        GBK_LAUNCHED();
        rc = cub_scan_excl(rowcount, f->merge_ptr, n + 1, s);
        if (rc) return rc;
        GBK_CUDA(cudaMalloc(&f->merge_idx, 4 * (nv > 0 ? nv : 1)));
        GBK_CUDA(cudaMemsetAsync(rowcount, 0, 4 * (n + 1), s));
        k_merge_fill<<<blocks_for(nv), 256, 0, s>>>(vrow, nv, f->merge_ptr, rowcount, f->merge_idx);
        GBK_LAUNCHED();
        k_merge_sort<<<blocks_for(n), 256, 0, s>>>(f->merge_ptr, n, f->merge_idx);
        GBK_LAUNCHED();
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(tmp);
        cudaFree(keys);
        cudaFree(keys2);
        cudaFree(pos);
        cudaFree(pos2);
        cudaFree(flag);
        cudaFree(vid);
        cudaFree(vrow);
        cudaFree(rowcount);
    } else {
        v.nrows = 0;
        GBK_CUDA(cudaMalloc(&v.ptr, 4));
        GBK_CUDA(cudaMemsetAsync(v.ptr, 0, 4, s));
        GBK_CUDA(cudaMalloc(&f->merge_idx, 4));
    }
    int rc = build_tiles(v, sizeof(T), s);
    if (rc) return rc;
    GBK_CUDA(cudaMalloc(&f->partial, sizeof(T) * (f->nvrows > 0 ? f->nvrows : 1)));
    GBK_CUDA(cudaStreamSynchronize(s));
    cudaFree(col_seg);
    return GBK_SUCCESS;
}

// Column degrees of one orientation, on the host (build-time only).
int host_col_degrees(const CsrView& a, std::vector<int64_t>& cdeg, cudaStream_t s) {
    std::vector<int32_t> idx(a.nnz);
    if (a.nnz) GBK_CUDA(cudaMemcpyAsync(idx.data(), a.idx, 4 * a.nnz, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    cdeg.assign(a.ncols, 0);
    for (int32_t c : idx) cdeg[c]++;
    return GBK_SUCCESS;
}

// CSR_SEG segmentation (seg_csr/build.hpp:34-105): segments of seg_cols
// columns; the smallest segments, until they hold >= 15 % of nnz, merge into
// segment 0 (the reference's __CSR_SEG_MERGE_SMALL__ rule).
template <typename T>
int build_seg(const CsrView& a, int32_t seg_cols, SegCsr** out, cudaStream_t s) {
    std::vector<int64_t> cdeg;
    int rc = host_col_degrees(a, cdeg, s);
    if (rc) return rc;
    const int64_t nseg0 = a.ncols > 0 ? (a.ncols - 1) / seg_cols + 1 : 1;
    std::vector<int64_t> est(nseg0, 0);
    for (int64_t c = 0; c < a.ncols; c++) est[c / seg_cols] += cdeg[c];
    std::vector<int64_t> order(nseg0);
    for (int64_t i = 0; i < nseg0; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return est[x] < est[y]; });
    std::vector<bool> small(nseg0, false);
    int64_t merged = 0;
    for (int64_t i = 0; i < nseg0; i++) {
        small[order[i]] = true;
        merged += est[order[i]];
        if (merged >= (int64_t)(0.15 * a.nnz)) break;
    }
    std::vector<int32_t> conv(nseg0);
    int32_t next = 1;
    for (int64_t i = 0; i < nseg0; i++) conv[i] = small[i] ? 0 : next++;
    std::vector<int32_t> col_seg(a.ncols);
    for (int64_t c = 0; c < a.ncols; c++) col_seg[c] = conv[c / seg_cols];
    SegCsr* f = new SegCsr();
    rc = build_segmented<T>(a, col_seg, nullptr, next, f, s);
    if (rc) return rc;
    *out = f;
    return GBK_SUCCESS;
}

// LAV with staged windows: the reference's column order (in-degree,
// descending; lav/build.hpp:113-141), computed on the device, and the
// renumbered matrix in the staged-window layout of CSR_SEG.  The renumbering
// packs the most used columns into the first windows -- the reference's
// "dense" segments (the columns holding dense_frac of nnz, lav/build.hpp:
// 143-160) -- so those windows are dense and each is staged once per CTA;
// the reference's one "sparse" segment becomes the remaining windows, staged
// the same way.  x is gathered into the new order on every call
// (spmv_lav.h:24-26).
}  // namespace

// Column order by in-degree, descending, ties in column order (the
// reference's LAV order, lav/build.hpp:113-141), computed on the device:
// *new_to_old (ncols) and the column ids relabelled into *idx_out (nnz), both
// allocated here (cudaMalloc, the caller frees them); *dense_cols = the
// first renumbered column at which the running in-degree sum reaches
// dense_frac of nnz.
int indegree_order(const CsrView& a, float dense_frac, int32_t** new_to_old, int32_t** idx_out,
                   int64_t* dense_cols, cudaStream_t s) {
    const int64_t nc = a.ncols, nnz = a.nnz;
    int32_t *cdeg = nullptr, *cdeg_sorted = nullptr, *iota = nullptr, *old_to_new = nullptr, *idx2 = nullptr,
            *n2o = nullptr;
    long long *acc = nullptr, *thr = nullptr;
    const int64_t nc1 = nc > 0 ? nc : 1;
    GBK_CUDA(cudaMalloc(&n2o, 4 * nc1));
    GBK_CUDA(cudaMalloc(&cdeg, 4 * nc1));
    GBK_CUDA(cudaMalloc(&cdeg_sorted, 4 * nc1));
    GBK_CUDA(cudaMalloc(&iota, 4 * nc1));
    GBK_CUDA(cudaMalloc(&old_to_new, 4 * nc1));
    GBK_CUDA(cudaMalloc(&idx2, 4 * (nnz > 0 ? nnz : 1)));
    GBK_CUDA(cudaMalloc(&acc, 8 * nc1));
    GBK_CUDA(cudaMalloc(&thr, 8));
    GBK_CUDA(cudaMemsetAsync(cdeg, 0, 4 * nc1, s));
    GBK_CUDA(cudaMemsetAsync(thr, 0, 8, s));
    const unsigned gs = (unsigned)std::min<int64_t>(blocks_for(nnz), 8 * num_sms());
    if (nnz > 0) {
        k_col_hist<<<blocks_for(nnz), 256, 0, s>>>(a.idx, nnz, cdeg);
        GBK_LAUNCHED();
    }
    if (nc > 0) {
        k_iota32<<<blocks_for(nc), 256, 0, s>>>(iota, nc);
        GBK_LAUNCHED();
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, cdeg, cdeg_sorted, iota, n2o, (int)nc, 0, 32, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, std::max<size_t>(tb, 16)));
        GBK_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp, tb, cdeg, cdeg_sorted, iota, n2o, (int)nc, 0, 32, s));
        count_launch(1);
        size_t sb = 0;
        cub::DeviceScan::InclusiveSum(nullptr, sb, cdeg_sorted, acc, (int)nc, s);
        void* stmp = nullptr;
        GBK_CUDA(cudaMalloc(&stmp, std::max<size_t>(sb, 16)));
        GBK_CUDA(cub::DeviceScan::InclusiveSum(stmp, sb, cdeg_sorted, acc, (int)nc, s));
        count_launch(1);
        k_dense_threshold<<<1, 1, 0, s>>>(acc, nc, (long long)(dense_frac * nnz), thr);
        GBK_LAUNCHED();
        k_invert_perm<<<blocks_for(nc), 256, 0, s>>>(n2o, nc, old_to_new);
        GBK_LAUNCHED();
        if (nnz > 0) {
            k_relabel<<<gs, 256, 0, s>>>(a.idx, nnz, old_to_new, idx2);
            GBK_LAUNCHED();
        }
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(tmp);
        cudaFree(stmp);
    }
    long long dc = 0;
    GBK_CUDA(cudaMemcpyAsync(&dc, thr, 8, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    cudaFree(cdeg);
    cudaFree(cdeg_sorted);
    cudaFree(iota);
    cudaFree(old_to_new);
    cudaFree(acc);
    cudaFree(thr);
    *new_to_old = n2o;
    *idx_out = idx2;
    if (dense_cols) *dense_cols = dc;
    return GBK_SUCCESS;
}

namespace {

int build_lav_staged(const CsrView& a, int dtype, float dense_frac, SegCsr** out, cudaStream_t s) {
    const int64_t nc = a.ncols;
    SegCsr* f = new SegCsr();
    f->n = a.nrows;
    f->ncols = nc;
    const size_t eb = dtype == GBK_F32 ? sizeof(float) : sizeof(int32_t);
    GBK_CUDA(cudaMalloc(&f->xr, eb * (nc > 0 ? nc : 1)));
    int32_t* idx2 = nullptr;
    int rc = indegree_order(a, dense_frac, &f->col_new_to_old, &idx2, &f->dense_cols, s);
    if (rc) {
        free_seg(f);
        return rc;
    }
    CsrView r = a;  // same rows and values, relabelled columns
    r.idx = idx2;
    r.bins = nullptr;
    rc = build_segsmem(r, dtype, &f->staged, s);
    cudaFree(idx2);
    if (rc) {
        free_seg(f);
        return rc;
    }
    *out = f;
    return GBK_SUCCESS;
}

// LAV (lav/build.hpp:97-212) without staging: columns renumbered by
// in-degree, descending; the columns holding the first dense_frac of nnz form
// "dense" segments of seg_cols columns, the rest one "sparse" segment; one
// segment-major virtual CSR and an in-order merge.
template <typename T>
int build_lav(const CsrView& a, int32_t seg_cols, float dense_frac, SegCsr** out, cudaStream_t s) {
    std::vector<int64_t> cdeg;
    int rc = host_col_degrees(a, cdeg, s);
    if (rc) return rc;
    std::vector<int32_t> new_to_old(a.ncols), old_to_new(a.ncols);
    for (int64_t c = 0; c < a.ncols; c++) new_to_old[c] = (int32_t)c;
    std::stable_sort(new_to_old.begin(), new_to_old.end(),
                     [&](int32_t x, int32_t y) { return cdeg[x] > cdeg[y]; });
    for (int64_t i = 0; i < a.ncols; i++) old_to_new[new_to_old[i]] = (int32_t)i;
    int64_t acc = 0, dense_threshold = 0;
    for (int64_t c = 0; c < a.ncols; c++) {
        acc += cdeg[new_to_old[c]];
        if (acc >= (int64_t)(dense_frac * a.nnz)) {
            dense_threshold = c;
            break;
        }
    }
    const int32_t ndense = dense_threshold > 0 ? (int32_t)((dense_threshold - 1) / seg_cols + 1) : 0;
    std::vector<int32_t> col_seg(a.ncols);
    for (int64_t c = 0; c < a.ncols; c++) {
        int32_t nc = old_to_new[c];
        col_seg[c] = nc < dense_threshold ? nc / seg_cols : ndense;
    }
    SegCsr* f = new SegCsr();
    GBK_CUDA(cudaMalloc(&f->col_new_to_old, 4 * (a.ncols > 0 ? a.ncols : 1)));
    GBK_CUDA(cudaMemcpyAsync(f->col_new_to_old, new_to_old.data(), 4 * a.ncols, cudaMemcpyHostToDevice, s));
    int32_t* old_to_new_d = nullptr;
    GBK_CUDA(cudaMalloc(&old_to_new_d, 4 * (a.ncols > 0 ? a.ncols : 1)));
    GBK_CUDA(cudaMemcpyAsync(old_to_new_d, old_to_new.data(), 4 * a.ncols, cudaMemcpyHostToDevice, s));
    rc = build_segmented<T>(a, col_seg, old_to_new_d, ndense + 1, f, s);
    cudaFree(old_to_new_d);
    if (rc) return rc;
    GBK_CUDA(cudaMalloc(&f->xr, sizeof(T) * (a.ncols > 0 ? a.ncols : 1)));
    *out = f;
    return GBK_SUCCESS;
}

// ---------------------------------------------------------------------------
// SpMV dispatch per format

template <int SR, typename T>
int run_sell(const SellC* f, int accum, const T* x, T* y, cudaStream_t s) {
    if (f->new_to_old) {  // renumbered columns: gather x into the new order first
        k_permute_x<T><<<blocks_for(f->ncols), 256, 0, s>>>(x, f->new_to_old, f->ncols, (T*)f->xr);
        GBK_LAUNCHED();
        x = (const T*)f->xr;
    }
    if (f->hot > 0) {
        const int smem = (int)(f->hot * sizeof(T));
        static bool attr_set = false;
        if (!attr_set) {
            GBK_CUDA(cudaFuncSetAttribute(k_sell_items_hot<SR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kMaxHotBytes));
            attr_set = true;
        }
        if (f->nitems > 0) {
            k_sell_items_hot<SR, T><<<(unsigned)num_sms(), kHotThreads, smem, s>>>(
                f->item_slice, f->item_j0, f->slice_item0, f->slice_len, f->slice_ptr, f->col, (const T*)f->val,
                f->perm, f->n, f->nitems, f->hot, x, y, accum, (T*)f->item_out, f->nreal, (T*)f->piece);
            GBK_LAUNCHED();
        }
    } else if (f->nitems > 0) {
        k_sell_items<SR, T><<<blocks_for(f->nitems * 32), 256, 0, s>>>(
            f->item_slice, f->item_j0, f->slice_item0, f->slice_len, f->slice_ptr, f->col, (const T*)f->val, f->perm,
            f->n, f->nitems, x, y, accum, (T*)f->item_out, f->nreal, (T*)f->piece);
        GBK_LAUNCHED();
    }
    if (f->nmulti > 0) {
        k_sell_fold<SR, T><<<blocks_for(f->nmulti * kSellC), 256, 0, s>>>(
            f->multi, f->nmulti, f->slice_item0, (const T*)f->item_out, f->perm, f->n, y, accum, f->nreal,
            (T*)f->piece);
        GBK_LAUNCHED();
    }
    if (f->nov > 0) {
        int rc = spmv_csr(f->ov, SR, GBK_OP_SECOND, dtype_of_t<T>(), x, f->ov_out, nullptr, 0, 0, s);
        if (rc) return rc;
        k_scatter_rows<T><<<blocks_for(f->nov), 256, 0, s>>>(f->ov_rows, (const T*)f->ov_out, f->nov, y, accum,
                                                             f->nreal, (T*)f->piece);
        GBK_LAUNCHED();
    }
    if (f->nlong > 0) {
        k_piece_fold<SR, T><<<blocks_for(f->nlong), 256, 0, s>>>(f->long_rows, f->long_p0, f->nlong,
                                                                 (const T*)f->piece, y, accum);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

template <int SR, typename T>
int run_seg(const SegCsr* f, int accum, const T* x, T* y, cudaStream_t s) {
    const T* xin = x;
    if (f->col_new_to_old) {
        k_reorder_x<T><<<blocks_for(f->ncols), 256, 0, s>>>(x, f->col_new_to_old, f->ncols, (T*)f->xr);
        GBK_LAUNCHED();
        xin = (const T*)f->xr;
    }
    if (f->staged) return run_segsmem(f->staged, SR, accum, dtype_of_t<T>(), xin, y, s);
    if (f->nvrows > 0) {
        int rc = spmv_csr(f->v, SR, GBK_OP_SECOND, dtype_of_t<T>(), xin, f->partial, nullptr, 0, 0, s);
        if (rc) return rc;
    }
    if (f->n > 0) {
        k_seg_merge<SR, T><<<blocks_for(f->n), 256, 0, s>>>(f->merge_ptr, f->merge_idx, (const T*)f->partial, f->n,
                                                            y, accum);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

template <typename T>
int format_dispatch(gbk_matrix A, int orient, int sr, int accum, const T* x, T* y, cudaStream_t s) {
#define FMT_CASE(SRV)                                                          \
    case SRV:                                                                  \
        if (A->format == GBK_FMT_SELL_C) return run_sell<SRV, T>(A->sell[orient], accum, x, y, s); \
        if (A->format == GBK_FMT_CSR_SEG) return run_seg<SRV, T>(A->seg[orient], accum, x, y, s);  \
        {                                                                      \
            const int rc = run_seg<SRV, T>(A->lav[orient], accum, x, y, s);    \
            if (rc != GBK_UNSUPPORTED) return rc;                              \
        }                                                                      \
        break;
    switch (sr) {
        FMT_CASE(GBK_PLUS_TIMES)
        FMT_CASE(GBK_LOR_LAND)
        FMT_CASE(GBK_FIRST_MIN)
        FMT_CASE(GBK_PLUS_SECOND)
        FMT_CASE(GBK_STRUCTURAL_BOOL)
        FMT_CASE(GBK_MIN_PLUS)
        FMT_CASE(GBK_MIN_SECOND)
        FMT_CASE(GBK_MIN_NOTEQ)
        FMT_CASE(GBK_PLUS_ONE)
        default:
            break;
    }
#undef FMT_CASE
    // non-associative add operators keep the reference's in-order CSR loop
    const CsrView& v = orient ? A->csc : A->csr;
    return spmv_csr(v, sr, accum, dtype_of_t<T>(), x, y, nullptr, 0, 0, s);
}

}  // namespace

int spmv_format(gbk_matrix A, int transpose, int sr, int accum, int dtype, const void* x, void* y,
                cudaStream_t s) {
    const int orient = transpose ? 1 : 0;
    if (A->format == GBK_FMT_SELL_C && A->sellw[orient]) {
        const int rc = run_sellw(A->sellw[orient], sr, accum, dtype, x, y, s);
        if (rc != GBK_UNSUPPORTED) return rc;
        return spmv_csr(orient ? A->csc : A->csr, sr, accum, dtype, x, y, nullptr, 0, 0, s);
    }
    if (A->format == GBK_FMT_CSR_SEG && A->segx[orient]) {
        const int rc = run_segsmem(A->segx[orient], sr, accum, dtype, x, y, s);
        if (rc != GBK_UNSUPPORTED) return rc;
        // add operators that cannot be folded atomically: the CSR kernels
        return spmv_csr(orient ? A->csc : A->csr, sr, accum, dtype, x, y, nullptr, 0, 0, s);
    }
    if (dtype == GBK_F32) return format_dispatch<float>(A, orient, sr, accum, (const float*)x, (float*)y, s);
    return format_dispatch<int32_t>(A, orient, sr, accum, (const int32_t*)x, (int32_t*)y, s);
}

int free_formats(gbk_matrix A) {
    for (int o = 0; o < 2; o++) {
        free_sell(A->sell[o]);
        free_seg(A->seg[o]);
        free_seg(A->lav[o]);
        free_segsmem(A->segx[o]);
        A->segx[o] = nullptr;
        free_sellw(A->sellw[o]);
        A->sellw[o] = nullptr;
        A->sell[o] = nullptr;
        A->seg[o] = nullptr;
        A->lav[o] = nullptr;
    }
    A->format = GBK_FMT_CSR;
    A->format_gen += 1;
    return GBK_SUCCESS;
}

int build_format(gbk_matrix A, gbk_format fmt, const gbk_format_params* p, cudaStream_t s) {
    gbk_format_params prm{};
    if (p) prm = *p;
    if (prm.sell_c == 0) prm.sell_c = kSellC;
    if (prm.sell_sigma == 0) prm.sell_sigma = 4096;
    if (prm.seg_cols == 0) prm.seg_cols = 131072;
    if (prm.lav_dense_frac == 0.0f) prm.lav_dense_frac = 0.8f;
    GBK_REQUIRE(prm.sell_hot_cols >= 0 && prm.sell_hot_cols * 4 <= kMaxHotBytes && prm.sell_hot_cols % 4 == 0,
                GBK_INVALID_VALUE, "sell_hot_cols %d: a multiple of 4 up to %d", prm.sell_hot_cols,
                kMaxHotBytes / 4);
    GBK_REQUIRE(prm.sell_c == kSellC, GBK_UNSUPPORTED, "SELL-C: slice height %d not provided (32 = one warp)",
                prm.sell_c);
    GBK_REQUIRE(prm.sell_sigma >= 1 && prm.seg_cols >= 1 && prm.lav_dense_frac > 0.0f && prm.lav_dense_frac <= 1.0f,
                GBK_INVALID_VALUE, "bad format parameters");
    GBK_REQUIRE(prm.csr_kernel >= 0 && prm.csr_kernel <= kKernelChunks, GBK_INVALID_VALUE, "bad csr_kernel %d",
                prm.csr_kernel);
    GBK_REQUIRE(prm.seg_staged >= -1 && prm.seg_staged <= 1, GBK_INVALID_VALUE, "bad seg_staged %d",
                prm.seg_staged);
    free_formats(A);
    A->params = prm;
    A->csr.kernel = prm.csr_kernel;
    A->csc.kernel = prm.csr_kernel;
    if (fmt == GBK_FMT_CSR) return GBK_SUCCESS;
    GBK_REQUIRE(fmt == GBK_FMT_SELL_C || fmt == GBK_FMT_CSR_SEG || fmt == GBK_FMT_LAV, GBK_INVALID_VALUE,
                "unknown format %d", (int)fmt);
    int rc = ensure_csc(A, s);
    if (rc) return rc;
    for (int o = 0; o < 2; o++) {
        const CsrView& v = o ? A->csc : A->csr;
        if (fmt == GBK_FMT_SELL_C && prm.seg_staged == 1) {
            rc = build_sellw(v, A->vtype, prm.sell_reorder_cols != 0, &A->sellw[o], s);
        } else if (fmt == GBK_FMT_SELL_C) {
            rc = A->vtype == GBK_F32
                     ? build_sell<float>(v, prm.sell_sigma, prm.sell_hot_cols, prm.sell_reorder_cols, &A->sell[o], s)
                     : build_sell<int32_t>(v, prm.sell_sigma, prm.sell_hot_cols, prm.sell_reorder_cols, &A->sell[o],
                                           s);
        } else if (fmt == GBK_FMT_CSR_SEG && prm.seg_staged >= 0) {
            rc = build_segsmem(v, A->vtype, &A->segx[o], s);
        } else if (fmt == GBK_FMT_CSR_SEG) {
            rc = A->vtype == GBK_F32 ? build_seg<float>(v, prm.seg_cols, &A->seg[o], s)
                                     : build_seg<int32_t>(v, prm.seg_cols, &A->seg[o], s);
        } else if (prm.seg_staged >= 0) {
            rc = build_lav_staged(v, A->vtype, prm.lav_dense_frac, &A->lav[o], s);
        } else {
            rc = A->vtype == GBK_F32 ? build_lav<float>(v, prm.seg_cols, prm.lav_dense_frac, &A->lav[o], s)
                                     : build_lav<int32_t>(v, prm.seg_cols, prm.lav_dense_frac, &A->lav[o], s);
        }
        if (rc) return rc;
    }
    A->format = fmt;
    A->format_gen += 1;
    return GBK_SUCCESS;
}

size_t format_bytes(gbk_matrix A) {
    size_t b = 0;
    const size_t eb = dtype_size(A->vtype);
    for (int o = 0; o < 2; o++) {
        if (A->sell[o]) {
            const SellC* f = A->sell[o];
            b += f->padded * (4 + eb) + f->nslices * 12 + f->n * 4 + f->nov * (4 + eb);
            b += f->ov.nnz * (4 + eb) + (f->ov.nrows + 1) * 4;
        }
        b += segsmem_bytes(A->segx[o]);
        b += sellw_bytes(A->sellw[o]);
        const SegCsr* g = A->seg[o] ? A->seg[o] : A->lav[o];
        if (g && g->staged) b += segsmem_bytes(g->staged) + g->ncols * (4 + eb);
        else if (g) b += g->v.nnz * (4 + eb) + (g->nvrows + 1) * 4 * 2 + (g->n + 1) * 4 + g->nvrows * eb;
    }
    return b;
}

int64_t format_padded_nnz(gbk_matrix A) {
    if (A->format == GBK_FMT_SELL_C && A->sell[0]) return A->sell[0]->padded + A->sell[0]->ov.nnz;
    if (A->format == GBK_FMT_SELL_C && A->sellw[0]) return sellw_padded(A->sellw[0]);
    return A->csr.nnz;
}

}  // namespace gbk

extern "C" int gbk_matrix_set_format(gbk_matrix A, gbk_format fmt, const gbk_format_params* params, void* stream) {
    GBK_REQUIRE(A, GBK_NULL_POINTER, "gbk_matrix_set_format: NULL matrix");
    return gbk::build_format(A, fmt, params, (cudaStream_t)stream);
}
