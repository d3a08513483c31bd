// Push SpMSpV and sparse-mask SpMV.
//
// SpMSpV replaces backend::SpMSpV with its three push kernels
// (src/backend/spmspv/spmspv.h:103-158, spmspv_atomics.h:5-170): for every
// frontier entry (i, x_i) scatter mul(A, x_i) into y.  The reference gives
// each OpenMP thread frontier vertices and updates y with `omp atomic`,
// plain stores or an `omp critical` section per edge.  Here the work unit is
// an edge: a scan of the frontier degrees turns the frontier into one flat
// edge range, cut into warp tiles of 256 consecutive edges, so a hub vertex
// is spread over many warps.  Per tile the warp finds the frontier entry of
// the tile's first edge (a 32-way search, one load per lane per round); per
// 32-edge sub-tile the lanes load the next 32 entry boundaries and each lane
// finds its own entry by a 5-step search over those boundaries in registers
// (shuffles).  Updates are warp-aggregated:
// lanes whose edges hit the same output element (match-any on the index)
// combine their values with the semiring's add in a tree over the group,
// and one lane per group issues the atomic (add; min on integers, a CAS loop
// on floats).  Or-monoids store 1 without an atomic, as the reference does.
#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr int kPushThreads = 256;
constexpr int kPushItems = 4;

__device__ __forceinline__ void atomic_min_val(int32_t* p, int32_t v) { atomicMin(p, v); }
__device__ __forceinline__ void atomic_min_val(float* p, float v) {
    int32_t* ip = (int32_t*)p;
    int32_t old = *ip;
    while (v < __int_as_float(old)) {
        int32_t prev = atomicCAS(ip, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
}

__global__ void k_frontier_degrees(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ids, int64_t nf,
                                   int32_t* __restrict__ deg) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < nf) deg[k] = ptr[ids[k] + 1] - ptr[ids[k]];
    if (k == nf) deg[k] = 0;
}

// Bit position of the r-th (0-based) set bit of m (m has more than r bits).
__device__ __forceinline__ int nth_set_bit(unsigned m, int r) {
    int pos = 0;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1)
        if (__popc(m & ((1u << (pos + w)) - 1u)) <= r) pos += w;
    return pos;
}

template <int SR, typename T>
__device__ __forceinline__ void push_atomic(int probe, T* y, int32_t j, T v) {
    using S = Semiring<SR, T>;
    if (probe == 8)
        atomicAdd(y + j, v);
    else  // min-monoids (min, first-min, min-plus, min-second, min-noteq)
        atomic_min_val(y + j, S::add(Lim<T>::max(), v));
}

// Largest k in [0, nf) with offs[k] <= e (offs ascending, offs[nf] > e),
// found by the whole warp: each round the 31 lanes probe 31 evenly spaced
// entries of the open range and a ballot keeps the sub-range, so a frontier
// of n entries takes about log32(n) rounds of one load each.
__device__ __forceinline__ int64_t warp_find_entry(const int32_t* __restrict__ offs, int64_t nf, int64_t e,
                                                   int lane) {
    int64_t lo = 0, hi = nf;  // offs[lo] <= e < offs[hi] (offs[nf] = E > e)
    while (hi - lo > 1) {
        const int64_t span = hi - lo;
        const int64_t p = lo + (span * (lane + 1) + 31) / 32;  // lanes 0..30 probe inside (lo, hi]
        const bool le = lane < 31 && p < hi && offs[p] <= e;
        const unsigned bal = __ballot_sync(0xffffffffu, le);
        const int c = __popc(bal);  // a prefix of the lanes (offs ascends)
        const int64_t p_c = __shfl_sync(0xffffffffu, p, c < 31 ? c : 30);
        const int64_t p_last = __shfl_sync(0xffffffffu, p, c > 0 ? c - 1 : 0);
        if (c > 0) lo = p_last;
        if (c < 31) hi = p_c;
    }
    return lo;
}

constexpr int kPushSubTiles = 8;  // 32-edge sub-tiles per warp tile

// One warp per tile of 256 consecutive frontier edges (grid-stride over
// tiles; the loops are warp-uniform, so every shuffle sees all 32 lanes).
// The tile's first entry comes from one warp search; each 32-edge sub-tile
// starts from the entry of the previous sub-tile's last edge.
template <int SR, typename T>
__global__ void __launch_bounds__(kPushThreads) k_push(const int32_t* __restrict__ ptr,
                                                       const int32_t* __restrict__ idx, const T* __restrict__ val,
                                                       const int32_t* __restrict__ ids, const T* __restrict__ xv,
                                                       int64_t nf, const int32_t* __restrict__ offs, int probe,
                                                       T* __restrict__ y) {
    using S = Semiring<SR, T>;
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int64_t kTile = 32 * kPushSubTiles;
    const int lane = threadIdx.x & 31;
    const int64_t E = offs[nf];
    const int64_t ntiles = (E + kTile - 1) / kTile;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; t < ntiles; t += nwarps) {
        int64_t k0 = warp_find_entry(offs, nf, t * kTile, lane);
        for (int sub = 0; sub < kPushSubTiles; ++sub) {
            const int64_t e0 = t * kTile + 32 * sub;
            if (e0 >= E) break;
            const int32_t start0 = offs[k0];
            // boundary of entry k0 + 1 + lane (E past the last entry)
            const int64_t kb = k0 + 1 + lane;
            const int32_t b = kb <= nf ? offs[kb] : (int32_t)E;
            const int64_t e = e0 + lane;
            const bool valid = e < E;
            // cnt = boundaries <= e among the 32 (they ascend with the lane)
            int cnt = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int32_t bv = __shfl_sync(kFull, b, cnt + step - 1);
                if (bv <= e) cnt += step;
            }
            const int32_t b31 = __shfl_sync(kFull, b, 31);
            const int32_t prev = __shfl_sync(kFull, b, cnt > 0 ? cnt - 1 : 0);
            int64_t k;
            int32_t start;
            if (valid && cnt == 31 && b31 <= e) {
                // more than 32 entries end before this edge (empty rows): search on
                int64_t lo = k0 + 32, hi = nf;
                while (hi - lo > 1) {
                    const int64_t mid = (lo + hi) >> 1;
                    if (offs[mid] <= e)
                        lo = mid;
                    else
                        hi = mid;
                }
                k = lo;
                start = offs[k];
            } else {
                k = k0 + cnt;  // an entry of the frontier for every valid lane
                start = cnt > 0 ? prev : start0;
            }
            int32_t j = -1 - lane;  // a key no other lane has
            T m = S::identity();
            if (valid) {
                const int32_t src = ids[k];
                const int64_t pos = ptr[src] + (e - start);
                j = idx[pos];
                m = S::mul(val[pos], xv[k]);
            }
            if (probe == 1) {
                if (valid) y[j] = T(1);
            } else if (SR != GBK_FIRST_WINS) {
                // first(y, m) == y leaves y unchanged; every other add folds per group
                const unsigned peers = __match_any_sync(kFull, j);
                const int rank = __popc(peers & ((1u << lane) - 1u));
                const int gsize = __popc(peers);
                T acc = m;
                for (int st = 1; st < 32; st <<= 1) {
                    if (!__any_sync(kFull, gsize > st)) break;
                    const bool take = (rank % (2 * st)) == 0 && rank + st < gsize;
                    const int from = take ? nth_set_bit(peers, rank + st) : lane;
                    const T o = __shfl_sync(kFull, acc, from);
                    if (take) acc = S::add(acc, o);
                }
                if (valid && rank == 0) push_atomic<SR, T>(probe, y, j, acc);
            }
            // the next sub-tile starts in the entry of this one's last edge
            // (valid whenever a next sub-tile exists: e0 + 32 < E)
            k0 = __shfl_sync(kFull, k, 31);
        }
    }
}

template <typename T>
__global__ void k_fill_t(T* y, int64_t n, T v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = v;
}

// apply_mask (spmspv.h:17-99), dense form (sparse complements are expanded first)
template <typename T>
__global__ void k_apply_mask_dense(T* y, const T* old, int64_t n, int accum, const void* m, int mdt, int mmode) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        bool sel = mask_selects(m, mdt, mmode, i);
        y[i] = sel ? binop<T>(accum, old[i], y[i]) : T(0);
    }
}

template <typename T>
__global__ void k_apply_mask_ids(T* y, const T* old, const int32_t* ids, int64_t nv, int accum) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nv; k += (int64_t)gridDim.x * blockDim.x) {
        int32_t i = ids[k];
        y[i] = binop<T>(accum, old[i], y[i]);
    }
}

__global__ void k_mark(const int32_t* ids, int64_t nv, uint8_t* flag) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nv; k += (int64_t)gridDim.x * blockDim.x)
        flag[ids[k]] = 1;
}

// One warp per listed row (SpMV_sparse without complement).
template <int SR, typename T>
__global__ void k_spmv_rows(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const T* __restrict__ val, const int32_t* __restrict__ rows, int64_t nr,
                            const T* __restrict__ x, T* __restrict__ y, int accum) {
    using S = Semiring<SR, T>;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = warp; k < nr; k += nwarps) {
        const int32_t r = rows[k];
        T acc = S::identity();
        if constexpr (Semiring<SR, T>::assoc) {
            for (int e = ptr[r] + lane; e < ptr[r + 1]; e += 32) acc = S::add(acc, S::mul(val[e], x[idx[e]]));
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc = S::add(acc, __shfl_down_sync(0xffffffffu, acc, off));
        } else {
            if (lane == 0)
                for (int e = ptr[r]; e < ptr[r + 1]; e++) acc = S::add(acc, S::mul(val[e], x[idx[e]]));
        }
        if (lane == 0) y[r] = (accum == GBK_OP_SECOND) ? acc : binop<T>(accum, y[r], acc);
    }
}

inline unsigned grid_cap(int64_t work, int threads) {
    int64_t b = (work + threads - 1) / threads;
    int64_t cap = (int64_t)num_sms() * 8;
    if (b > cap) b = cap;
    return (unsigned)(b > 0 ? b : 1);
}

template <typename T>
int spmspv_t(int sr, const CsrView& v, int accum, const int32_t* ids, const void* xv, int64_t nf, T* y,
             const gbk_mask* mask, cudaStream_t s) {
    const int64_t n = v.nrows == v.ncols ? v.ncols : v.ncols;  // y is indexed by the pushed-to side
    const int probe = semiring_probe(sr, 0);
    T ident;
    switch (sr) {
        case GBK_MIN_PLUS:
        case GBK_CUSTOM_LESS_PLUS:
        case GBK_MIN_SECOND:
        case GBK_MIN_NOTEQ:
            ident = Lim<T>::max();
            break;
        default:
            ident = T(0);
    }
    T* old = nullptr;
    if (mask) {
        GBK_CUDA(cudaMallocAsync((void**)&old, sizeof(T) * (n > 0 ? n : 1), s));
        GBK_CUDA(cudaMemcpyAsync(old, y, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
    }
    if (n > 0) {
        k_fill_t<T><<<grid_cap(n, 256), 256, 0, s>>>(y, n, ident);
        GBK_LAUNCHED();
    }
    if (nf > 0) {
        int32_t *deg = nullptr, *offs = nullptr;
        GBK_CUDA(cudaMallocAsync((void**)&deg, sizeof(int32_t) * (nf + 1), s));
        GBK_CUDA(cudaMallocAsync((void**)&offs, sizeof(int32_t) * (nf + 1), s));
        k_frontier_degrees<<<(unsigned)((nf + 1 + 255) / 256), 256, 0, s>>>(v.ptr, ids, nf, deg);
        GBK_LAUNCHED();
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, offs, (int)(nf + 1), s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMallocAsync(&tmp, tb, s));
        GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, deg, offs, (int)(nf + 1), s));
        count_launch(1);
        const unsigned grid = (unsigned)num_sms() * 8;
#define PUSH_CASE(SRV)                                                                                          \
    case SRV:                                                                                                   \
        k_push<SRV, T><<<grid, kPushThreads, 0, s>>>(v.ptr, v.idx, (const T*)v.val, ids, (const T*)xv, nf, offs, \
                                                     probe, y);                                                 \
        break;
        switch (sr) {
            PUSH_CASE(GBK_PLUS_TIMES)
            PUSH_CASE(GBK_LOR_LAND)
            PUSH_CASE(GBK_FIRST_WINS)
            PUSH_CASE(GBK_FIRST_MIN)
            PUSH_CASE(GBK_PLUS_SECOND)
            PUSH_CASE(GBK_STRUCTURAL_BOOL)
            PUSH_CASE(GBK_MIN_PLUS)
            PUSH_CASE(GBK_CUSTOM_LESS_PLUS)
            PUSH_CASE(GBK_MIN_SECOND)
            PUSH_CASE(GBK_MIN_NOTEQ)
            PUSH_CASE(GBK_PLUS_ONE)
            default:
                set_error("gbk_spmspv: unknown semiring %d", sr);
                return GBK_INVALID_VALUE;
        }
#undef PUSH_CASE
        GBK_LAUNCHED();
        cudaFreeAsync(tmp, s);
        cudaFreeAsync(deg, s);
        cudaFreeAsync(offs, s);
    }
    if (mask && n > 0) {
        if (mask->dense) {
            k_apply_mask_dense<T><<<grid_cap(n, 256), 256, 0, s>>>(y, old, n, accum, mask->dense, mask->dtype,
                                                                   mask->mode);
            GBK_LAUNCHED();
        } else if (mask->mode == GBK_MASK_STR_COMP) {
            uint8_t* flag = nullptr;
            GBK_CUDA(cudaMallocAsync((void**)&flag, n, s));
            GBK_CUDA(cudaMemsetAsync(flag, 0, n, s));
            if (mask->nvals > 0) {
                k_mark<<<grid_cap(mask->nvals, 256), 256, 0, s>>>(mask->ids, mask->nvals, flag);
                GBK_LAUNCHED();
            }
            k_apply_mask_dense<T><<<grid_cap(n, 256), 256, 0, s>>>(y, old, n, accum, flag, GBK_BOOL,
                                                                   GBK_MASK_STR_COMP);
            GBK_LAUNCHED();
            cudaFreeAsync(flag, s);
        } else if (mask->nvals > 0) {
            k_apply_mask_ids<T><<<grid_cap(mask->nvals, 256), 256, 0, s>>>(y, old, mask->ids, mask->nvals, accum);
            GBK_LAUNCHED();
        }
    }
    if (old) cudaFreeAsync(old, s);
    return GBK_SUCCESS;
}

template <typename T>
int rows_t(int sr, const CsrView& v, int accum, const T* x, T* y, const int32_t* rows, int64_t nr, cudaStream_t s) {
    if (nr == 0) return GBK_SUCCESS;
    const unsigned grid = grid_cap(nr * 32, 256);
#define ROWS_CASE(SRV)                                                                                    \
    case SRV:                                                                                             \
        k_spmv_rows<SRV, T><<<grid, 256, 0, s>>>(v.ptr, v.idx, (const T*)v.val, rows, nr, x, y, accum); \
        break;
    switch (sr) {
        ROWS_CASE(GBK_PLUS_TIMES)
        ROWS_CASE(GBK_LOR_LAND)
        ROWS_CASE(GBK_FIRST_WINS)
        ROWS_CASE(GBK_FIRST_MIN)
        ROWS_CASE(GBK_PLUS_SECOND)
        ROWS_CASE(GBK_STRUCTURAL_BOOL)
        ROWS_CASE(GBK_MIN_PLUS)
        ROWS_CASE(GBK_CUSTOM_LESS_PLUS)
        ROWS_CASE(GBK_MIN_SECOND)
        ROWS_CASE(GBK_MIN_NOTEQ)
        ROWS_CASE(GBK_PLUS_ONE)
        default:
            set_error("unknown semiring %d", sr);
            return GBK_INVALID_VALUE;
    }
#undef ROWS_CASE
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

}  // namespace

}  // namespace gbk

using namespace gbk;

extern "C" {

int gbk_spmspv(gbk_matrix A, int transpose, gbk_semiring sr, gbk_binop accum, gbk_dtype dtype,
               const int32_t* x_ids, const void* x_vals, int64_t x_nvals, void* y, const gbk_mask* mask,
               void* stream) {
    GBK_REQUIRE(A && y, GBK_NULL_POINTER, "gbk_spmspv: NULL argument");
    GBK_REQUIRE(x_nvals == 0 || (x_ids && x_vals), GBK_NULL_POINTER, "gbk_spmspv: NULL frontier");
    GBK_REQUIRE(dtype == A->vtype, GBK_DOMAIN_MISMATCH, "gbk_spmspv: vector type %d != matrix type %d", (int)dtype,
                (int)A->vtype);
    cudaStream_t s = (cudaStream_t)stream;
    // mxv pushes along columns of A (the CSC), vxm along rows (the CSR): spmspv.h:125-146
    if (!transpose) {
        int rc = ensure_csc(A, s);
        if (rc) return rc;
    }
    const CsrView& v = transpose ? A->csr : A->csc;
    if (dtype == GBK_F32) return spmspv_t<float>(sr, v, accum, x_ids, x_vals, x_nvals, (float*)y, mask, s);
    if (dtype == GBK_I32) return spmspv_t<int32_t>(sr, v, accum, x_ids, x_vals, x_nvals, (int32_t*)y, mask, s);
    set_error("gbk_spmspv: element type %d unsupported", (int)dtype);
    return GBK_UNSUPPORTED;
}

int gbk_mxv_sparse_mask(gbk_matrix A, int transpose, gbk_semiring sr, gbk_binop accum, gbk_dtype dtype,
                        const void* x, void* y, const int32_t* mask_ids, int64_t mask_nvals, gbk_mask_mode mask_mode,
                        void* stream) {
    GBK_REQUIRE(A && x && y, GBK_NULL_POINTER, "gbk_mxv_sparse_mask: NULL argument");
    GBK_REQUIRE(mask_nvals == 0 || mask_ids, GBK_NULL_POINTER, "gbk_mxv_sparse_mask: NULL mask ids");
    GBK_REQUIRE(dtype == A->vtype, GBK_DOMAIN_MISMATCH, "gbk_mxv_sparse_mask: type mismatch");
    cudaStream_t s = (cudaStream_t)stream;
    if (transpose) {
        int rc = ensure_csc(A, s);
        if (rc) return rc;
    }
    const CsrView& v = transpose ? A->csc : A->csr;
    if (mask_mode == GBK_MASK_STR_COMP) {  // spmv_csr.h:218-255: densify, complement
        uint8_t* flag = nullptr;
        const int64_t n = v.nrows;
        GBK_CUDA(cudaMallocAsync((void**)&flag, n > 0 ? n : 1, s));
        GBK_CUDA(cudaMemsetAsync(flag, 0, n > 0 ? n : 1, s));
        if (mask_nvals > 0) {
            k_mark<<<grid_cap(mask_nvals, 256), 256, 0, s>>>(mask_ids, mask_nvals, flag);
            GBK_LAUNCHED();
        }
        int rc = spmv_csr(v, sr, accum, dtype, x, y, flag, GBK_BOOL, GBK_MASK_STR_COMP, s);
        cudaFreeAsync(flag, s);
        return rc;
    }
    if (dtype == GBK_F32) return rows_t<float>(sr, v, accum, (const float*)x, (float*)y, mask_ids, mask_nvals, s);
    if (dtype == GBK_I32)
        return rows_t<int32_t>(sr, v, accum, (const int32_t*)x, (int32_t*)y, mask_ids, mask_nvals, s);
    set_error("gbk_mxv_sparse_mask: element type %d unsupported", (int)dtype);
    return GBK_UNSUPPORTED;
}

}  // extern "C"
