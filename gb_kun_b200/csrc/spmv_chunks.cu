// CSR SpMV over equal runs of entries: one warp per 256 consecutive entries
// of the CSR arrays, whatever rows they fall in.
//
// Each lane takes 8 consecutive entries (two 16-byte loads of column ids and
// two of values, streamed), gathers their x values, finds the row of its
// first entry by a binary search of the row pointers between the chunk's
// first and last rows, and walks its entries: a row that begins and ends
// inside the lane is written at once; the lane's first and last partial
// sums go through one segmented warp scan keyed by row, so a row spread over
// several lanes is summed inside the warp and written by the lane holding
// its last entry.  A row that crosses a chunk boundary leaves its part of
// each chunk in a per-chunk slot (its first chunk: `tail`, every later one:
// `head`), and a second kernel adds them in chunk order.  Rows without
// entries are listed at build time and receive the identity.  Each row's sum
// is formed in a fixed order, so results repeat bit for bit.
//
// No work depends on row lengths, so a hub row of 10^5 entries costs the
// same per entry as a row of one, and every warp issues its loads at once
// (no per-row loop whose depth grows with the row).  Same computation as
// SpMV_all_active_diff_vectors (src/backend/spmv/spmv_csr.h:340-384), with
// the reference's nnz-balanced thread ranges (src/helpers/balancing/
// balancing.h:5-33) cut at warp granularity instead of per OpenMP thread.
#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr int kChunk = 256;      // entries per warp
constexpr int kLane = 8;         // entries per lane
constexpr int kThreads = 256;    // 8 warps per CTA
constexpr int kWarpsPerCta = kThreads / 32;

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<int32_t> { using type = int4; };

// 8 consecutive elements from a 32-byte aligned address, evict-first.
template <typename T>
__device__ __forceinline__ void ld8(const T* p, T (&v)[kLane]) {
    using V = typename Vec4<T>::type;
    const V a = __ldcs(reinterpret_cast<const V*>(p));
    const V b = __ldcs(reinterpret_cast<const V*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

template <typename T>
__device__ __forceinline__ void put(T* y, int32_t r, T v, int accum, const void* mask, int mdt, int mmode) {
    if (mask && !mask_selects(mask, mdt, mmode, r)) {
        y[r] = T(0);  // outside the mask (spmv_csr.h:324-327)
        return;
    }
    y[r] = (accum == GBK_OP_SECOND) ? v : binop<T>(accum, y[r], v);
}

template <int SR, typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_chunks(
    const int32_t* __restrict__ rptr, const int32_t* __restrict__ rows, const int32_t* __restrict__ idx,
    const T* __restrict__ val, int64_t nnz, int64_t nchunks, const int32_t* __restrict__ chunk_k,
    const int32_t* __restrict__ empty_rows, int64_t nempty, const T* __restrict__ x, T* __restrict__ y, int accum,
    const void* mask, int mdt, int mmode, T* __restrict__ head, T* __restrict__ tail) {
    using S = Semiring<SR, T>;
    const int64_t chunk_ctas = (nchunks + kWarpsPerCta - 1) / kWarpsPerCta;
    if ((int64_t)blockIdx.x >= chunk_ctas) {  // rows without entries
        const int64_t i = ((int64_t)blockIdx.x - chunk_ctas) * kThreads + threadIdx.x;
        if (i < nempty) put<T>(y, empty_rows[i], S::identity(), accum, mask, mdt, mmode);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (w >= nchunks) return;  // the whole warp leaves together
    const int32_t base = (int32_t)(w * kChunk);
    const int64_t end64 = (int64_t)base + kChunk < nnz ? (int64_t)base + kChunk : nnz;
    const int32_t end = (int32_t)end64;
    const int32_t e0 = base + lane * kLane;
    const int nv = max(0, min(kLane, end - e0));  // entries of this lane

    // the lane's entries and their products
    int32_t c[kLane];
    T a[kLane], xv[kLane];
    if (nv == kLane) {
        ld8<int32_t>(idx + e0, c);
        ld8<T>(val + e0, a);
    } else {
#pragma unroll
        for (int j = 0; j < kLane; j++) {
            c[j] = j < nv ? ld_stream(idx + e0 + j) : 0;
            a[j] = j < nv ? ld_stream(val + e0 + j) : T(0);
        }
    }
    // gathers first: their latency overlaps the row search below
    const uint64_t pol = policy_evict_last();
#pragma unroll
    for (int j = 0; j < kLane; j++) xv[j] = j < nv ? ld_keep(x + c[j], pol) : T(0);

    // row (index among the rows with entries) of the first entry:
    // lo + #{q in (lo, hi] : rptr[q] <= e0}, counted over windows of 32 row
    // starts (one coalesced load each; a chunk of rows averaging 8+ entries
    // needs one) by a 5-step shuffle search per lane
    const int32_t lo = chunk_k[w], hi = chunk_k[w + 1];
    const int32_t last_e0 = end - 1 - ((end - 1 - base) % kLane);  // first entry of the last busy lane
    int32_t cnt = 0;
    for (int32_t wb = lo + 1;; wb += 32) {
        const int32_t q = wb + lane;
        const int32_t P = q <= hi ? __ldg(rptr + q) : INT32_MAX;
        int k = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
            if (__shfl_sync(0xffffffffu, P, k + step - 1) <= e0) k += step;
        const int32_t P31 = __shfl_sync(0xffffffffu, P, 31);
        if (k == 31 && P31 <= e0) k = 32;
        cnt += k;
        if (P31 > last_e0) break;  // later windows start rows after every lane's first entry
    }
    int32_t kr = lo + cnt, rbeg = 0, rend = 0;
    if (nv > 0) {
        rbeg = __ldg(rptr + kr);
        rend = __ldg(rptr + kr + 1);
    }

    // walk: rows that begin and end inside the lane are written here; rows
    // with entries are consecutive in rptr, so the next entry's row is the
    // next one
    const int32_t kA = kr;
    T sA = S::identity(), acc = S::identity();
    bool closedA = false;  // the first row ends inside this lane, before its last entry
#pragma unroll
    for (int j = 0; j < kLane; j++) {
        if (j < nv) {
            const int32_t e = e0 + j;
            if (e >= rend) {
                if (!closedA) {
                    sA = acc;
                    closedA = true;
                } else {
                    put<T>(y, __ldg(rows + kr), acc, accum, mask, mdt, mmode);
                }
                acc = S::identity();
                kr++;
                rend = __ldg(rptr + kr + 1);
            }
            acc = S::add(acc, S::mul(a[j], xv[j]));
        }
    }
    if (!closedA) sA = acc;
    const bool openL = nv > 0 && rbeg < e0;      // the first row began in an earlier lane or chunk
    const bool openR = nv > 0 && rend > e0 + nv;  // the last row goes on after this lane
    if (nv > 0 && closedA) {
        if (!openL) put<T>(y, __ldg(rows + kA), sA, accum, mask, mdt, mmode);
        if (!openR) put<T>(y, __ldg(rows + kr), acc, accum, mask, mdt, mmode);
    } else if (nv > 0 && !openL && !openR) {
        put<T>(y, __ldg(rows + kA), sA, accum, mask, mdt, mmode);
    }

    // segmented scan of the last-row partials: a lane whose only row began
    // earlier continues the previous lane's sum, every other lane starts one
    T sc = acc;
    int flag = !(nv > 0 && !closedA && openL);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T su = __shfl_up_sync(0xffffffffu, sc, d);
        const int fu = __shfl_up_sync(0xffffffffu, flag, d);
        if (lane >= d) {
            if (!flag) sc = S::add(su, sc);
            flag |= fu;
        }
    }
    const T cin = __shfl_up_sync(0xffffffffu, sc, 1);
    // the lane holding the last entry of a row that began in an earlier lane
    if (openL && (closedA || !openR)) {
        const T total = lane > 0 ? S::add(cin, sA) : sA;
        if (rbeg < base) head[w] = total;  // began in an earlier chunk: the fix-up adds it
        else put<T>(y, __ldg(rows + kA), total, accum, mask, mdt, mmode);
    }
    // the chunk's last row goes on into the next chunk
    if (openR && e0 + nv == end) {
        const bool began_before = !closedA && rbeg < base;
        if (began_before) head[w] = sc;
        else tail[w] = sc;
    }
}

// Rows that cross a chunk boundary, summed from their per-chunk parts in a
// fixed order.  One thread per chunk boundary c takes the row that begins in
// chunk c-1 and goes on into chunk c, when it touches at most kLongSpan
// chunks: its first chunk's part, then each later chunk's part in order.
// Rows over more chunks (listed at build time) take a warp each after those
// threads: lane-strided partial sums over the chunks, then a fixed
// shuffle tree.
constexpr int kLongSpan = 32;

template <int SR, typename T>
__global__ void k_spmv_chunks_fixup(const int32_t* __restrict__ rptr, const int32_t* __restrict__ rows,
                                    int64_t nchunks, const int32_t* __restrict__ chunk_k,
                                    const int32_t* __restrict__ long_k, int64_t nlong, const T* __restrict__ head,
                                    const T* __restrict__ tail, T* __restrict__ y, int accum, const void* mask,
                                    int mdt, int mmode) {
    using S = Semiring<SR, T>;
    const int64_t boundary_ctas = (nchunks - 1 + 255) / 256;
    if ((int64_t)blockIdx.x >= boundary_ctas) {  // long rows: a warp each
        const int lane = threadIdx.x & 31;
        const int64_t i = ((int64_t)blockIdx.x - boundary_ctas) * (blockDim.x / 32) + (threadIdx.x >> 5);
        if (i >= nlong) return;  // the whole warp leaves together
        const int32_t k = long_k[i];
        const int64_t c0 = rptr[k] / kChunk, c1 = ((int64_t)rptr[k + 1] - 1) / kChunk;
        T acc = S::identity();
        for (int64_t c = c0 + lane; c <= c1; c += 32) acc = S::add(acc, c == c0 ? tail[c] : head[c]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc = S::add(acc, __shfl_xor_sync(0xffffffffu, acc, off));
        if (lane == 0) put<T>(y, rows[k], acc, accum, mask, mdt, mmode);
        return;
    }
    const int64_t c = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    const int32_t k = chunk_k[c];
    const int64_t b = rptr[k];
    if (b >= c * kChunk || b < (c - 1) * kChunk) return;  // not a row that begins in chunk c-1
    const int64_t last = ((int64_t)rptr[k + 1] - 1) / kChunk;
    if (last - (c - 1) + 1 > kLongSpan) return;  // a long row: its warp sums it
    T acc = tail[c - 1];
#pragma unroll 8
    for (int64_t q = c; q <= last; q++) acc = S::add(acc, head[q]);
    put<T>(y, rows[k], acc, accum, mask, mdt, mmode);
}

// Build: rows with entries (ascending) and their starts, rows without.
__global__ void k_row_flags(const int32_t* __restrict__ ptr, int64_t n, int32_t* __restrict__ flag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) flag[i] = ptr[i + 1] > ptr[i] ? 1 : 0;
}

__global__ void k_row_split(const int32_t* __restrict__ ptr, int64_t n, const int32_t* __restrict__ flag,
                            const int32_t* __restrict__ pos, int32_t* __restrict__ rows,
                            int32_t* __restrict__ rptr, int32_t* __restrict__ empty_rows,
                            int32_t* __restrict__ counts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t k = pos[i];
    if (flag[i]) {
        rows[k] = (int32_t)i;
        rptr[k] = ptr[i];
    } else {
        empty_rows[i - k] = (int32_t)i;
    }
    if (i == n - 1) {
        const int32_t m = k + flag[i];
        rptr[m] = ptr[n];
        counts[0] = m;
        counts[1] = (int32_t)(n - m);
    }
}

__global__ void k_chunk_k(const int32_t* __restrict__ rptr, int64_t m, int64_t nnz, int64_t nchunks,
                          int32_t* __restrict__ chunk_k) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c > nchunks) return;
    const int64_t e = c * kChunk < nnz ? c * kChunk : nnz - 1;
    int64_t lo = 0, hi = m - 1;  // the largest k with rptr[k] <= e
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (rptr[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    chunk_k[c] = (int32_t)lo;
}

__global__ void k_long_rows(const int32_t* __restrict__ rptr, int64_t m, int32_t* __restrict__ list,
                            int32_t* __restrict__ count) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool is_long = false;
    if (k < m) {
        const int64_t c0 = rptr[k] / kChunk, c1 = ((int64_t)rptr[k + 1] - 1) / kChunk;
        is_long = c1 - c0 + 1 > kLongSpan;
    }
    const unsigned bits = __ballot_sync(0xffffffffu, is_long);
    if (!bits) return;
    const int lane = threadIdx.x & 31;
    int32_t first = 0;
    if (lane == __ffs(bits) - 1) first = atomicAdd(count, __popc(bits));
    first = __shfl_sync(0xffffffffu, first, __ffs(bits) - 1);
    if (is_long) list[first + __popc(bits & ((1u << lane) - 1))] = (int32_t)k;
}

}  // namespace

struct RowChunks {
    int64_t nchunks = 0, nrows_nz = 0, nempty = 0, nlong = 0;
    int32_t* rows = nullptr;        // rows with entries, ascending (nrows_nz)
    int32_t* rptr = nullptr;        // their starts, then nnz (nrows_nz + 1)
    int32_t* empty_rows = nullptr;  // rows without entries
    int32_t* chunk_k = nullptr;     // per chunk: index in rows of the row holding its first entry (nchunks + 1)
    int32_t* long_k = nullptr;      // rows over more than kLongSpan chunks (indices in rows)
    void* head = nullptr;           // nchunks elements each
    void* tail = nullptr;
};

void free_chunks(RowChunks* c) {
    if (!c) return;
    cudaFree(c->rows);
    cudaFree(c->rptr);
    cudaFree(c->empty_rows);
    cudaFree(c->chunk_k);
    cudaFree(c->long_k);
    cudaFree(c->head);
    cudaFree(c->tail);
    delete c;
}

bool chunks_usable(const CsrView& v) {
    return ((uintptr_t)v.idx % 16) == 0 && ((uintptr_t)v.val % 16) == 0;
}

namespace {

// Stream-ordered temporaries released on every return path.
struct Scratch {
    cudaStream_t s;
    void* p[4] = {nullptr, nullptr, nullptr, nullptr};
    explicit Scratch(cudaStream_t st) : s(st) {}
    ~Scratch() {
        for (void* q : p)
            if (q) cudaFreeAsync(q, s);
    }
};

int fill_chunks(const CsrView& v, int elem_bytes, RowChunks* rc, cudaStream_t s) {
    const int64_t n = v.nrows, nnz = v.nnz;
    rc->nchunks = (nnz + kChunk - 1) / kChunk;
    Scratch sc(s);
    size_t tb = 0;
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, (const int32_t*)nullptr, (int32_t*)nullptr, (int)n, s));
    for (int i = 0; i < 4; i++) GBK_CUDA(cudaMallocAsync(&sc.p[i], i == 2 ? 12 : i == 3 ? tb : 4 * (size_t)n, s));
    int32_t *flag = (int32_t*)sc.p[0], *pos = (int32_t*)sc.p[1], *counts = (int32_t*)sc.p[2];
    GBK_CUDA(cudaMemsetAsync(counts, 0, 12, s));
    GBK_CUDA(cudaMalloc(&rc->rows, 4 * n));
    GBK_CUDA(cudaMalloc(&rc->rptr, 4 * (n + 1)));
    GBK_CUDA(cudaMalloc(&rc->empty_rows, 4 * n));
    GBK_CUDA(cudaMalloc(&rc->long_k, 4 * n));
    const unsigned g = (unsigned)((n + 255) / 256);
    k_row_flags<<<g, 256, 0, s>>>(v.ptr, n, flag);
    GBK_LAUNCHED();
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(sc.p[3], tb, flag, pos, (int)n, s));
    count_launch(1);
    k_row_split<<<g, 256, 0, s>>>(v.ptr, n, flag, pos, rc->rows, rc->rptr, rc->empty_rows, counts);
    GBK_LAUNCHED();
    int32_t h[3] = {0, 0, 0};
    GBK_CUDA(cudaMemcpyAsync(h, counts, 8, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    rc->nrows_nz = h[0];
    rc->nempty = h[1];
    if (rc->nchunks > 0) {
        GBK_CUDA(cudaMalloc(&rc->chunk_k, 4 * (rc->nchunks + 1)));
        GBK_CUDA(cudaMalloc(&rc->head, (size_t)elem_bytes * rc->nchunks));
        GBK_CUDA(cudaMalloc(&rc->tail, (size_t)elem_bytes * rc->nchunks));
        k_chunk_k<<<(unsigned)((rc->nchunks + 1 + 255) / 256), 256, 0, s>>>(rc->rptr, rc->nrows_nz, nnz,
                                                                            rc->nchunks, rc->chunk_k);
        GBK_LAUNCHED();
        k_long_rows<<<(unsigned)((rc->nrows_nz + 255) / 256), 256, 0, s>>>(rc->rptr, rc->nrows_nz, rc->long_k,
                                                                           counts + 2);
        GBK_LAUNCHED();
        GBK_CUDA(cudaMemcpyAsync(h + 2, counts + 2, 4, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        rc->nlong = h[2];
    }
    return GBK_SUCCESS;
}

}  // namespace

int build_chunks(const CsrView& v, int elem_bytes, RowChunks** out, cudaStream_t s) {
    GBK_REQUIRE(chunks_usable(v), GBK_INVALID_VALUE, "entry-chunk SpMV: column / value arrays not 16-byte aligned");
    GBK_REQUIRE(v.nrows > 0, GBK_INVALID_VALUE, "entry-chunk SpMV: no rows");
    RowChunks* rc = new RowChunks();
    const int st = fill_chunks(v, elem_bytes, rc, s);
    if (st != GBK_SUCCESS) {
        free_chunks(rc);
        return st;
    }
    *out = rc;
    return GBK_SUCCESS;
}

template <int SR, typename T>
int spmv_chunks_t(const RowChunks* rc, const CsrView& v, int accum, const T* x, T* y, const void* mask, int mdt,
                  int mmode, cudaStream_t s) {
    const int64_t ctas = (rc->nchunks + kWarpsPerCta - 1) / kWarpsPerCta + (rc->nempty + kThreads - 1) / kThreads;
    if (ctas > 0) {
        k_spmv_chunks<SR, T><<<(unsigned)ctas, kThreads, 0, s>>>(
            rc->rptr, rc->rows, v.idx, (const T*)v.val, v.nnz, rc->nchunks, rc->chunk_k, rc->empty_rows,
            rc->nempty, x, y, accum, mask, mdt, mmode, (T*)rc->head, (T*)rc->tail);
        GBK_LAUNCHED();
    }
    if (rc->nchunks > 1) {
        const int64_t fctas = (rc->nchunks - 1 + 255) / 256 + (rc->nlong + 7) / 8;
        k_spmv_chunks_fixup<SR, T><<<(unsigned)fctas, 256, 0, s>>>(rc->rptr, rc->rows, rc->nchunks, rc->chunk_k,
                                                                  rc->long_k, rc->nlong, (const T*)rc->head,
                                                                  (const T*)rc->tail, y, accum, mask, mdt, mmode);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

template <typename T>
int spmv_chunks_dispatch(const RowChunks* rc, const CsrView& v, int sr, int accum, const T* x, T* y,
                         const void* mask, int mdt, int mmode, cudaStream_t s) {
    switch (sr) {
        case GBK_PLUS_TIMES: return spmv_chunks_t<GBK_PLUS_TIMES, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_LOR_LAND: return spmv_chunks_t<GBK_LOR_LAND, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_FIRST_MIN: return spmv_chunks_t<GBK_FIRST_MIN, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_PLUS_SECOND: return spmv_chunks_t<GBK_PLUS_SECOND, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_STRUCTURAL_BOOL:
            return spmv_chunks_t<GBK_STRUCTURAL_BOOL, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_PLUS: return spmv_chunks_t<GBK_MIN_PLUS, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_SECOND: return spmv_chunks_t<GBK_MIN_SECOND, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_NOTEQ: return spmv_chunks_t<GBK_MIN_NOTEQ, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
        case GBK_PLUS_ONE: return spmv_chunks_t<GBK_PLUS_ONE, T>(rc, v, accum, x, y, mask, mdt, mmode, s);
    }
    set_error("entry-chunk SpMV: semiring %d not associative", sr);
    return GBK_UNSUPPORTED;
}

int spmv_chunks(const RowChunks* rc, const CsrView& v, int sr, int accum, int dtype, const void* x, void* y,
                const void* mask, int mdt, int mmode, cudaStream_t s) {
    if (dtype == GBK_F32)
        return spmv_chunks_dispatch<float>(rc, v, sr, accum, (const float*)x, (float*)y, mask, mdt, mmode, s);
    return spmv_chunks_dispatch<int32_t>(rc, v, sr, accum, (const int32_t*)x, (int32_t*)y, mask, mdt, mmode, s);
}

}  // namespace gbk
