// CSR SpMV over a semiring: merge-path tiles, one CTA per tile.
//
// Replaces SpMV_all_active_diff_vectors / _same_vectors / SpMV_dense
// (src/backend/spmv/spmv_csr.h:266-486).  The reference gives each OpenMP
// thread an nnz-balanced row range (src/helpers/balancing/balancing.h:5-33)
// and reduces each row serially.  On the GPU the unit of balance is a tile
// of kTileItems items of the merged list (row ends, nonzeros): every CTA gets
// the same amount of work whatever the degree skew, so hub rows of 10^5
// entries and runs of empty rows cost the same as average rows.
//
// Per tile:
//   1. stage the tile's row ends and the products mul(A_ij, x_j) in shared
//      memory (coalesced streaming loads of col/val, x gathered through L2);
//   2. each thread walks kSpmvItems merge items, closing rows as it meets
//      their ends;
//   3. a block-wide segmented scan hands each thread the partial sum of the
//      row it started in; rows that close inside the tile are written with
//      coalesced stores;
//   4. rows crossing tile boundaries leave a per-tile carry and are finished
//      by a small fix-up kernel in a fixed order (deterministic results).
// Non-associative "monoids" of the reference (first, less) are reduced row
// by row in order instead, exactly like the reference loop.
#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr unsigned kFull = 0xffffffffu;

template <typename T>
__device__ __forceinline__ void write_row(T* y, int64_t r, T v, int accum, const void* mask, int mdt, int mmode) {
    if (mask && !mask_selects(mask, mdt, mmode, r)) {
        y[r] = T(0);  // spmv_csr.h:324-327
        return;
    }
    y[r] = (accum == GBK_OP_SECOND) ? v : binop<T>(accum, y[r], v);
}

template <int SR, typename T>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv_merge(
    const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, const T* __restrict__ val,
    const int2* __restrict__ tiles, const T* __restrict__ x, T* __restrict__ y, int accum, const void* mask,
    int mdt, int mmode, int32_t* __restrict__ carry_row, T* __restrict__ carry_val, T* __restrict__ head_val) {
    using S = Semiring<SR, T>;
    __shared__ int32_t s_rowend[kTileItems + 1];
    __shared__ T s_prod[kTileItems];
    __shared__ T s_out[kTileItems];
    __shared__ T s_incl[kSpmvThreads];
    __shared__ int32_t s_wkey[kSpmvThreads / 32];
    __shared__ T s_wval[kSpmvThreads / 32];
    __shared__ int32_t s_pkey[kSpmvThreads / 32];
    __shared__ T s_pval[kSpmvThreads / 32];

    const int tile = blockIdx.x;
    const int2 c0 = tiles[tile];
    const int2 c1 = tiles[tile + 1];
    const int row0 = c0.x, nz0 = c0.y;
    const int nrow = c1.x - c0.x;
    const int nnzt = c1.y - c0.y;
    const int tid = threadIdx.x;

    // 1. stage row ends and products
    for (int k = tid; k < nrow; k += kSpmvThreads) s_rowend[k] = ld_stream(ptr + row0 + k + 1);
    if (tid == 0) s_rowend[nrow] = INT_MAX;
    {
        int c[kSpmvItems];
        T a[kSpmvItems];
#pragma unroll
        for (int i = 0; i < kSpmvItems; i++) {
            int k = tid + i * kSpmvThreads;
            if (k < nnzt) {
                c[i] = ld_stream(idx + nz0 + k);
                a[i] = ld_stream(val + nz0 + k);
            }
        }
        const uint64_t pol = policy_evict_last();
#pragma unroll
        for (int i = 0; i < kSpmvItems; i++) {
            int k = tid + i * kSpmvThreads;
            if (k < nnzt) s_prod[k] = S::mul(a[i], ld_keep(x + c[i], pol));
        }
    }
    __syncthreads();

    // 2. merge-path walk of this thread's items
    const int tile_items = nrow + nnzt;
    const int d = min(tid * kSpmvItems, tile_items);
    int lo = max(0, d - nnzt), hi = min(d, nrow);
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (s_rowend[mid] <= nz0 + d - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    int ti = lo, tj = d - lo;
    const int ti_start = ti;
    const int nitems = min(kSpmvItems, tile_items - d);
    T acc = S::identity();
    bool emitted = false;
#pragma unroll
    for (int k = 0; k < kSpmvItems; k++) {
        if (k < nitems) {
            if (s_rowend[ti] <= nz0 + tj) {
                s_out[ti] = acc;
                acc = S::identity();
                ti++;
                emitted = true;
            } else {
                acc = S::add(acc, s_prod[tj]);
                tj++;
            }
        }
    }

    // 3. block-wide segmented inclusive scan of (row in progress, partial)
    const int lane = tid & 31, warp = tid >> 5;
    int key = ti;
    T v = acc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int k2 = __shfl_up_sync(kFull, key, off);
        T v2 = __shfl_up_sync(kFull, v, off);
        if (lane >= off && k2 == key) v = S::add(v2, v);
    }
    if (lane == 31) {
        s_wkey[warp] = key;
        s_wval[warp] = v;
    }
    __syncthreads();
    if (tid == 0) {  // exclusive prefix over warp aggregates
        int pk = -1;
        T pv = S::identity();
        for (int w = 0; w < kSpmvThreads / 32; w++) {
            s_pkey[w] = pk;
            s_pval[w] = pv;
            if (s_wkey[w] == pk)
                pv = S::add(pv, s_wval[w]);
            else
                pv = s_wval[w];
            pk = s_wkey[w];
        }
    }
    __syncthreads();
    // The earlier warps' prefix carries key == this thread's key only when every
    // lane from the warp start to here is inside that same row: add it.
    if (warp > 0 && s_pkey[warp] == key) v = S::add(s_pval[warp], v);
    s_incl[tid] = v;
    __syncthreads();
    if (tid > 0 && emitted && ti_start < nrow) s_out[ti_start] = S::add(s_incl[tid - 1], s_out[ti_start]);
    if (tid == kSpmvThreads - 1) {
        carry_row[tile] = row0 + key;
        carry_val[tile] = v;
    }
    __syncthreads();

    // 4. rows closed in this tile
    const bool continued = nrow > 0 && nz0 > ld_stream(ptr + row0);
    for (int k = tid; k < nrow; k += kSpmvThreads) {
        if (k == 0 && continued) {
            head_val[tile] = s_out[0];
            continue;
        }
        write_row<T>(y, (int64_t)row0 + k, s_out[k], accum, mask, mdt, mmode);
    }
}

// Rows that crossed tiles: head part of the closing tile plus the carries of
// every earlier tile that ended inside the same row.
template <int SR, typename T>
__global__ void k_spmv_fixup(const int32_t* __restrict__ ptr, const int2* __restrict__ tiles, int64_t ntiles,
                             T* __restrict__ y, int accum, const void* mask, int mdt, int mmode,
                             const int32_t* __restrict__ carry_row, const T* __restrict__ carry_val,
                             const T* __restrict__ head_val) {
    using S = Semiring<SR, T>;
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int2 c0 = tiles[t], c1 = tiles[t + 1];
    if (c1.x - c0.x < 1 || c0.y <= ptr[c0.x]) return;
    const int r = c0.x;
    T total = head_val[t];
    for (int64_t k = t - 1; k >= 0 && carry_row[k] == r; k--) total = S::add(carry_val[k], total);
    write_row<T>(y, r, total, accum, mask, mdt, mmode);
}

// In-order row reduction for the reference's non-associative add operators.
template <int SR, typename T>
__global__ void k_spmv_rowseq(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                              const T* __restrict__ val, int64_t nrows, const T* __restrict__ x, T* __restrict__ y,
                              int accum, const void* mask, int mdt, int mmode) {
    using S = Semiring<SR, T>;
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    if (mask && !mask_selects(mask, mdt, mmode, r)) {
        y[r] = T(0);
        return;
    }
    T acc = S::identity();
    for (int e = ptr[r]; e < ptr[r + 1]; e++) acc = S::add(acc, S::mul(val[e], x[idx[e]]));
    y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
}

template <int SR, typename T>
int launch(const CsrView& v, int accum, const void* x, void* y, const void* mask, int mdt, int mmode,
           cudaStream_t s) {
    if (v.nrows == 0) return GBK_SUCCESS;
    if constexpr (!Semiring<SR, T>::assoc) {
        k_spmv_rowseq<SR, T><<<(unsigned)((v.nrows + 255) / 256), 256, 0, s>>>(
            v.ptr, v.idx, (const T*)v.val, v.nrows, (const T*)x, (T*)y, accum, mask, mdt, mmode);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    } else {
        static bool carveout_set = false;  // all shared memory for the tile buffers: 8 CTAs per SM
        if (!carveout_set) {
            GBK_CUDA(cudaFuncSetAttribute(k_spmv_merge<SR, T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared));
            carveout_set = true;
        }
        k_spmv_merge<SR, T><<<(unsigned)v.ntiles, kSpmvThreads, 0, s>>>(
            v.ptr, v.idx, (const T*)v.val, v.tile_coord, (const T*)x, (T*)y, accum, mask, mdt, mmode, v.carry_row,
            (T*)v.carry_val, (T*)v.head_val);
        GBK_LAUNCHED();
        if (v.ntiles > 1) {
            k_spmv_fixup<SR, T><<<(unsigned)((v.ntiles + 255) / 256), 256, 0, s>>>(
                v.ptr, v.tile_coord, v.ntiles, (T*)y, accum, mask, mdt, mmode, v.carry_row, (const T*)v.carry_val,
                (const T*)v.head_val);
            GBK_LAUNCHED();
        }
        return GBK_SUCCESS;
    }
}

template <typename T>
int dispatch(const CsrView& v, int sr, int accum, const void* x, void* y, const void* mask, int mdt, int mmode,
             cudaStream_t s) {
    switch (sr) {
        case GBK_PLUS_TIMES: return launch<GBK_PLUS_TIMES, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_LOR_LAND: return launch<GBK_LOR_LAND, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_FIRST_WINS: return launch<GBK_FIRST_WINS, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_FIRST_MIN: return launch<GBK_FIRST_MIN, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_PLUS_SECOND: return launch<GBK_PLUS_SECOND, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_STRUCTURAL_BOOL: return launch<GBK_STRUCTURAL_BOOL, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_PLUS: return launch<GBK_MIN_PLUS, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_CUSTOM_LESS_PLUS: return launch<GBK_CUSTOM_LESS_PLUS, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_SECOND: return launch<GBK_MIN_SECOND, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_MIN_NOTEQ: return launch<GBK_MIN_NOTEQ, T>(v, accum, x, y, mask, mdt, mmode, s);
        case GBK_PLUS_ONE: return launch<GBK_PLUS_ONE, T>(v, accum, x, y, mask, mdt, mmode, s);
    }
    set_error("unknown semiring %d", sr);
    return GBK_INVALID_VALUE;
}

}  // namespace

constexpr int64_t kChunksAutoNnz = 1ll << 23;

static bool assoc_semiring(int sr) { return sr != GBK_FIRST_WINS && sr != GBK_CUSTOM_LESS_PLUS; }

int spmv_csr(const CsrView& v, int sr, int accum, int dtype, const void* x, void* y, const void* mask,
             int mask_dtype, int mask_mode, cudaStream_t s) {
    GBK_REQUIRE(dtype == GBK_F32 || dtype == GBK_I32, GBK_UNSUPPORTED,
                "spmv: element type %d unsupported (GBK_F32 or GBK_I32)", dtype);
    // the default kernel: degree bins, except unmasked products over large
    // matrices, where equal runs of entries measured faster (R-MAT: 0.248
    // against 0.28 ms at 65 M entries, 65 against 72 us at 16 M, slower at
    // 4 M); a mask keeps the bins, which skip masked-out rows before any load
    const bool auto_chunks = v.kernel == kKernelAuto && !mask && v.nnz >= kChunksAutoNnz;
    if ((v.kernel == kKernelChunks || auto_chunks) && assoc_semiring(sr) && v.nrows > 0 && chunks_usable(v)) {
        if (!v.chunks) {
            int rc = build_chunks(v, (int)dtype_size(dtype), &v.chunks, s);
            if (rc) return rc;
        }
        return spmv_chunks(v.chunks, v, sr, accum, dtype, x, y, mask, mask_dtype, mask_mode, s);
    }
    if (v.kernel != kKernelMerge && assoc_semiring(sr) && v.nrows > 0) {
        if (!v.bins) {
            int rc = build_bins(v, (int)dtype_size(dtype), &v.bins, s);
            if (rc) return rc;
        }
        return spmv_binned(v.bins, v, sr, accum, dtype, x, y, mask, mask_dtype, mask_mode, s);
    }
    if (dtype == GBK_F32) return dispatch<float>(v, sr, accum, x, y, mask, mask_dtype, mask_mode, s);
    if (dtype == GBK_I32) return dispatch<int32_t>(v, sr, accum, x, y, mask, mask_dtype, mask_mode, s);
    set_error("spmv: element type %d unsupported (GBK_F32 or GBK_I32)", dtype);
    return GBK_UNSUPPORTED;
}

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_mxv(gbk_matrix A, int transpose, gbk_semiring sr, gbk_binop accum, gbk_dtype dtype,
                       const void* x, void* y, const void* mask, gbk_dtype mask_dtype, gbk_mask_mode mask_mode,
                       void* stream) {
    GBK_REQUIRE(A && x && y, GBK_NULL_POINTER, "gbk_mxv: NULL argument");
    GBK_REQUIRE(dtype == A->vtype, GBK_DOMAIN_MISMATCH, "gbk_mxv: vector type %d != matrix type %d", (int)dtype,
                (int)A->vtype);
    GBK_REQUIRE((int)accum >= 0 && (int)accum <= GBK_OP_ONE, GBK_INVALID_VALUE, "gbk_mxv: bad accumulator %d",
                (int)accum);
    cudaStream_t s = (cudaStream_t)stream;
    if (transpose) {
        int rc = ensure_csc(A, s);
        if (rc) return rc;
    }
    const CsrView& v = transpose ? A->csc : A->csr;
    const size_t eb = dtype_size(dtype);
    if (x == (const void*)y) {  // same vector in and out: read from a copy (spmv_csr.h:432-486)
        if (A->xcopy_elems < v.ncols) {
            cudaFree(A->xcopy);
            A->xcopy = nullptr;
            GBK_CUDA(cudaMalloc(&A->xcopy, eb * (v.ncols > 0 ? v.ncols : 1)));
            A->xcopy_elems = v.ncols;
        }
        GBK_CUDA(cudaMemcpyAsync(A->xcopy, x, eb * v.ncols, cudaMemcpyDeviceToDevice, s));
        x = A->xcopy;
    }
    if (!mask && A->format != GBK_FMT_CSR) return spmv_format(A, transpose, sr, accum, dtype, x, y, s);
    return spmv_csr(v, sr, accum, dtype, x, y, mask, mask_dtype, mask_mode, s);
}
