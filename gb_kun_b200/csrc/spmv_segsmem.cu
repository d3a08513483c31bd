// CSR_SEG SpMV with the x segment staged in shared memory.
//
// The reference's segmented CSR (src/backend/matrix/seg_csr/build.hpp:23-169,
// src/backend/spmv/spmv_seg.h:8-308) cuts the columns into windows so each
// segment's slice of x stays in cache, computes per-segment row sums and then
// merges them.  Here a window is kSegCols columns, the size of x that fits a
// CTA's shared memory (192 KiB of 4-byte values):
//   * the entries are re-sorted segment-major (then by row, then column), each
//     with a 16-bit column inside its window; a bit per entry marks the start
//     of a "virtual row" (the entries of one row inside one segment);
//   * 148 persistent CTAs (one per SM, 1024 threads) take equal shares of the
//     entries; for each segment it touches a CTA copies that window of x into
//     shared memory once, and its warps walk 32-entry chunks of their share:
//     coalesced 2-byte column / 4-byte value loads, the x gather from shared
//     memory, a segmented warp scan along the row-start bits;
//   * each virtual row's sum goes straight into y with one atomic of the
//     semiring's add (float / int add, int / float minimum, or a store of 1
//     for the logical-or semirings), so there is no merge pass.
// Float sums therefore add in an order that varies between runs (within the
// FP32 tolerance); integer and min / or results are exact.  Semirings whose
// add is not associative fall back to the CSR kernels.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace gbk {

constexpr int kSegCols = 49152;  // x values per staged window (192 KiB of 4-byte values)
constexpr int kSegThreads = 1024;
constexpr int kSegUnroll = 4;    // 32-entry chunks whose loads a warp keeps in flight

struct SegSmem {
    int64_t nrows = 0, ncols = 0, nnz = 0, nvrows = 0;
    int32_t nseg = 0;
    uint16_t* col = nullptr;       // column inside the window, nnz
    void* val = nullptr;           // nnz
    uint32_t* head = nullptr;      // one bit per entry: starts a virtual row (nnz padded to 32)
    int32_t* chunk_vr = nullptr;   // virtual row containing entry 32 k
    int32_t* vrow = nullptr;       // original row of each virtual row
    int32_t* seg_start = nullptr;  // nseg + 1 entry offsets
    void* tmp = nullptr;           // nrows: the product before the accumulator
    int32_t* err = nullptr;        // first out-of-range index seen by the kernel (0 = none)
    bool check = true;             // read err back after the first launch
};

namespace {

__global__ void k_ss_keys(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, int64_t n,
                          unsigned long long* __restrict__ keys, int32_t* __restrict__ pos) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    for (int32_t e = ptr[r]; e < ptr[r + 1]; ++e) {
        keys[e] = ((unsigned long long)(idx[e] / kSegCols) << 32) | (unsigned long long)r;
        pos[e] = e;
    }
}

template <typename T>
__global__ void k_ss_fill(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ pos,
                          const int32_t* __restrict__ idx, const T* __restrict__ v, int64_t nnz, int64_t padded,
                          uint16_t* __restrict__ col, T* __restrict__ val, int32_t* __restrict__ flag,
                          uint32_t* __restrict__ head, int32_t* __restrict__ seg_start) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // padded is a multiple of 32
    if (i >= padded) return;
    bool h = false;
    if (i < nnz) {
        const unsigned long long k = keys[i];
        const int32_t seg = (int32_t)(k >> 32);
        const int32_t e = pos[i];
        col[i] = (uint16_t)(idx[e] - seg * kSegCols);
        val[i] = v[e];
        h = (i == 0) || (keys[i - 1] != k);
        flag[i] = h;
        if (i == 0 || (int32_t)(keys[i - 1] >> 32) != seg) seg_start[seg] = (int32_t)i;
    }
    const unsigned w = __ballot_sync(0xffffffffu, h);
    if ((threadIdx.x & 31) == 0) head[i >> 5] = w;
}

__global__ void k_ss_vrows(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ flag,
                           const int32_t* __restrict__ vid, int64_t nnz, int32_t* __restrict__ vrow,
                           int32_t* __restrict__ chunk_vr) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    if (flag[i]) vrow[vid[i]] = (int32_t)(keys[i] & 0xffffffffu);
    if ((i & 31) == 0) chunk_vr[i >> 5] = vid[i] + flag[i] - 1;
}

// atomic fold of one virtual row's sum into out[r] by the semiring's add
template <int SR, typename T>
__device__ __forceinline__ void fold_into(T* out, int32_t r, T v);

__device__ __forceinline__ void atomic_min_any(float* p, float v) {
    // order-preserving on the bit patterns: non-negative floats order as ints,
    // negative ones in reverse as unsigned ints
    if (v >= 0.0f)
        atomicMin((int*)p, __float_as_int(v));
    else
        atomicMax((unsigned int*)p, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_min_any(int32_t* p, int32_t v) { atomicMin(p, v); }

__device__ __forceinline__ void atomic_add_any(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_any(int32_t* p, int32_t v) {
    // saturating, like elem_add, so INT_MAX stays the min-plus infinity
    int old = *((volatile int*)p), assumed;
    do {
        assumed = old;
        old = atomicCAS(p, assumed, elem_add(assumed, v));
    } while (old != assumed);
}

template <int SR>
struct AddClass {  // 0 plus, 1 min, 2 or, -1 not folded atomically
    static constexpr int value = (SR == GBK_PLUS_TIMES || SR == GBK_PLUS_SECOND || SR == GBK_PLUS_ONE) ? 0
                                 : (SR == GBK_MIN_PLUS || SR == GBK_MIN_SECOND || SR == GBK_FIRST_MIN ||
                                    SR == GBK_MIN_NOTEQ)
                                     ? 1
                                 : (SR == GBK_LOR_LAND || SR == GBK_STRUCTURAL_BOOL) ? 2
                                                                                      : -1;
};

template <int SR, typename T>
__device__ __forceinline__ void fold_into(T* out, int32_t r, T v) {
    using S = Semiring<SR, T>;
    constexpr int cls = AddClass<SR>::value;
    if constexpr (cls == 0) {
        if (v != T(0)) atomic_add_any(out + r, v);
    } else if constexpr (cls == 1) {
        if (v < S::identity()) atomic_min_any(out + r, v);
    } else {
        if (v != T(0)) out[r] = T(1);
    }
}

// One warp over entries [wa, wb) of the staged segment.
// Index checks: a virtual row, row or window column out of range is recorded
// in *err (first one wins) and the access skipped, so a malformed structure
// reports an error instead of touching memory it does not own.
__device__ __forceinline__ void ss_flag(int32_t* err, int32_t code) { atomicCAS(err, 0, code); }

template <int SR, typename T>
__device__ __forceinline__ void ss_warp_range(const uint16_t* __restrict__ col, const T* __restrict__ val,
                                              const uint32_t* __restrict__ head,
                                              const int32_t* __restrict__ chunk_vr,
                                              const int32_t* __restrict__ vrow, const T* xs, int w, int64_t wa,
                                              int64_t wb, T* out, int64_t nvrows, int64_t nrows,
                                              int32_t* err) {
    using S = Semiring<SR, T>;
    const unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned le = (lane == 31) ? kAll : ((2u << lane) - 1u);
    // the virtual row open just before entry wa
    const int64_t k = wa >> 5;
    const int b = (int)(wa & 31);
    const uint32_t hw = head[k];
    const int32_t vr_at_wa = chunk_vr[k] + __popc(hw & (b == 31 ? 0xfffffffeu : (((2u << b) - 1u) & ~1u)));
    int64_t vr_open = ((hw >> b) & 1) ? (int64_t)vr_at_wa - 1 : (int64_t)vr_at_wa;
    T carry = S::identity();
    for (int64_t e0 = wa; e0 < wb; e0 += 32 * kSegUnroll) {
        uint16_t cc[kSegUnroll];
        T vv[kSegUnroll];
        unsigned H[kSegUnroll];
#pragma unroll
        for (int u = 0; u < kSegUnroll; ++u) {
            const int64_t e = e0 + u * 32 + lane;
            const bool ok = e < wb;
            cc[u] = ok ? __ldcs(col + e) : (uint16_t)0;
            vv[u] = ok ? __ldcs(val + e) : T(0);
            const uint32_t hw = ok ? __ldg(head + (e >> 5)) : 0u;
            H[u] = __ballot_sync(kAll, ok && ((hw >> (e & 31)) & 1u));
        }
        // does the entry after this group start a virtual row?
        const int64_t en = e0 + 32 * kSegUnroll;
        const bool next_group_head = en < wb && ((__ldg(head + (en >> 5)) >> (en & 31)) & 1u);
        // the virtual rows these chunks touch are consecutive: fetch their row
        // ids together (lane j of chunk u holds virtual row vb[u] + off[u] + j)
        int32_t rr[kSegUnroll];
        int64_t vb[kSegUnroll];
        int off[kSegUnroll];
        {
            int64_t base = vr_open;
#pragma unroll
            for (int u = 0; u < kSegUnroll; ++u) {
                vb[u] = base;
                off[u] = (int)(H[u] & 1u);
                const int64_t q = base + off[u] + lane;
                rr[u] = (q >= 0 && q < nvrows) ? __ldg(vrow + q) : -1;
                base += __popc(H[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < kSegUnroll; ++u) {
            const int64_t eb = e0 + u * 32;
            if (eb >= wb) break;
            const int64_t e = eb + lane;
            const bool ok = e < wb;
            const bool in_win = cc[u] < w;
            if (ok && !in_win) ss_flag(err, 1);
            T v = (ok && in_win) ? S::mul(vv[u], xs[cc[u]]) : S::identity();
            const unsigned hle = H[u] & le;
            const int first = hle ? 31 - __clz(hle) : 0;  // first lane of this lane's run in the chunk
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const T o = __shfl_up_sync(kAll, v, d);
                if (lane - d >= first) v = S::add(v, o);
            }
            if (!hle) v = S::add(carry, v);  // the run continues the open virtual row
            const int j = __popc(hle);       // this run is virtual row vb[u] + j
            const int32_t r = __shfl_sync(kAll, rr[u], (j - off[u]) & 31);
            const int last = (int)min((int64_t)31, wb - 1 - eb);  // last valid lane of the chunk
            const bool next_head = lane < 31 && ((H[u] >> (lane + 1)) & 1u);
            // the run at `last` goes on into the next entry unless that starts a row
            bool cont = false;
            if (e + 1 < wb || eb + 32 < wb) {
                const bool nh = (u + 1 < kSegUnroll) ? (bool)(H[(u + 1) % kSegUnroll] & 1u) : next_group_head;
                cont = (last == 31) && (eb + 32 < wb) && !nh;
            }
            cont = __shfl_sync(kAll, cont, last);
            if (ok && (next_head || (lane == last && !cont))) {
                const int64_t vr = vb[u] + j;
                if (vr < 0 || vr >= nvrows || r < 0 || r >= nrows)
                    ss_flag(err, 2);
                else
                    fold_into<SR, T>(out, r, v);
            }
            carry = cont ? __shfl_sync(kAll, v, last) : S::identity();
        }
        {
#pragma unroll
            for (int u = 0; u < kSegUnroll; ++u) vr_open += __popc(H[u]);
        }
    }
}

template <int SR, typename T>
__global__ void __launch_bounds__(kSegThreads, 1)
    k_segsmem(const uint16_t* __restrict__ col, const T* __restrict__ val, const uint32_t* __restrict__ head,
              const int32_t* __restrict__ chunk_vr, const int32_t* __restrict__ vrow,
              const int32_t* __restrict__ seg_start, int32_t nseg, int64_t nnz, int64_t ncols, int64_t nvrows,
              int64_t nrows, const T* __restrict__ x, T* out, int32_t* err) {
    extern __shared__ __align__(16) unsigned char ss_smem[];
    T* xs = reinterpret_cast<T*>(ss_smem);
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int64_t c0 = nnz * blockIdx.x / gridDim.x, c1 = nnz * (blockIdx.x + 1) / gridDim.x;
    if (c0 >= c1) return;  // the whole block leaves together
    int lo = 0, hi = nseg;  // last segment starting at or before c0
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (seg_start[mid] <= c0)
            lo = mid;
        else
            hi = mid;
    }
    for (int s = lo; s < nseg && seg_start[s] < c1; ++s) {
        const int64_t a = max(c0, (int64_t)seg_start[s]), b = min(c1, (int64_t)seg_start[s + 1]);
        if (a >= b) continue;
        __syncthreads();  // the previous window's readers are done
        const int64_t col0 = (int64_t)s * kSegCols;
        const int w = (int)min((int64_t)kSegCols, ncols - col0);
        for (int i = threadIdx.x; i < w; i += blockDim.x) xs[i] = __ldg(x + col0 + i);
        __syncthreads();
        const int64_t nch = (b - a + 31) >> 5;
        const int64_t per = (nch + nwarps - 1) / nwarps;
        const int64_t wa = a + (int64_t)warp * per * 32;
        const int64_t wb = min(b, wa + per * 32);
        if (wa < wb) ss_warp_range<SR, T>(col, val, head, chunk_vr, vrow, xs, w, wa, wb, out, nvrows, nrows, err);
    }
}

template <typename T>
__global__ void k_ss_init(T* out, int64_t n, T v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v;
}

template <typename T>
__global__ void k_ss_accum(T* __restrict__ y, const T* __restrict__ t, int64_t n, int accum) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = binop<T>(accum, y[i], t[i]);
}

unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

template <typename T>
int build_impl(const CsrView& a, SegSmem** out, cudaStream_t s) {
    SegSmem* f = new SegSmem();
    f->nrows = a.nrows;
    f->ncols = a.ncols;
    f->nnz = a.nnz;
    f->nseg = (int32_t)std::max<int64_t>(1, (a.ncols + kSegCols - 1) / kSegCols);
    const int64_t nnz = a.nnz, padded = ((nnz + 31) / 32) * 32 + 32;
    auto fail = [&](int rc) {
        free_segsmem(f);
        return rc;
    };
    if (cudaMalloc(&f->col, 2 * std::max<int64_t>(nnz, 1)) || cudaMalloc(&f->val, sizeof(T) * std::max<int64_t>(nnz, 1)) ||
        cudaMalloc(&f->head, 4 * (padded / 32)) || cudaMalloc(&f->chunk_vr, 4 * (padded / 32)) ||
        cudaMalloc(&f->seg_start, 4 * (f->nseg + 1)) ||
        cudaMalloc(&f->tmp, sizeof(T) * std::max<int64_t>(a.nrows, 1)) || cudaMalloc(&f->err, 4))
        return fail(cuda_fail(cudaGetLastError(), "segmented format allocation", __FILE__, __LINE__));
    if (cudaMemsetAsync(f->head, 0, 4 * (padded / 32), s) || cudaMemsetAsync(f->chunk_vr, 0, 4 * (padded / 32), s) ||
        cudaMemsetAsync(f->err, 0, 4, s))
        return fail(cuda_fail(cudaGetLastError(), "cudaMemsetAsync", __FILE__, __LINE__));
    std::vector<int32_t> ss(f->nseg + 1, -1);
    if (nnz > 0) {
        unsigned long long *keys = nullptr, *keys2 = nullptr;
        int32_t *pos = nullptr, *pos2 = nullptr, *flag = nullptr, *vid = nullptr;
        GBK_CUDA(cudaMalloc(&keys, 8 * nnz));
        GBK_CUDA(cudaMalloc(&keys2, 8 * nnz));
        GBK_CUDA(cudaMalloc(&pos, 4 * nnz));
        GBK_CUDA(cudaMalloc(&pos2, 4 * nnz));
        GBK_CUDA(cudaMalloc(&flag, 4 * (nnz + 1)));
        GBK_CUDA(cudaMalloc(&vid, 4 * (nnz + 1)));
        k_ss_keys<<<blocks(a.nrows), 256, 0, s>>>(a.ptr, a.idx, a.nrows, keys, pos);
        GBK_LAUNCHED();
        int seg_bits = 1;
        while ((1ll << seg_bits) < f->nseg) ++seg_bits;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, pos, pos2, (int)nnz, 0, 32 + seg_bits, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, std::max<size_t>(tb, 16)));
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, pos, pos2, (int)nnz, 0, 32 + seg_bits, s));
        count_launch(1);
        GBK_CUDA(cudaMemsetAsync(f->seg_start, 0xff, 4 * (f->nseg + 1), s));
        GBK_CUDA(cudaMemsetAsync(flag + nnz, 0, 4, s));
        k_ss_fill<T><<<blocks(padded), 256, 0, s>>>(keys2, pos2, a.idx, (const T*)a.val, nnz, padded, f->col,
                                                    (T*)f->val, flag, f->head, f->seg_start);
        GBK_LAUNCHED();
        size_t sb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, sb, flag, vid, (int)(nnz + 1), s);
        void* stmp = nullptr;
        GBK_CUDA(cudaMalloc(&stmp, std::max<size_t>(sb, 16)));
        GBK_CUDA(cub::DeviceScan::ExclusiveSum(stmp, sb, flag, vid, (int)(nnz + 1), s));
        count_launch(1);
        int32_t nv = 0;
        GBK_CUDA(cudaMemcpyAsync(&nv, vid + nnz, 4, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaMemcpyAsync(ss.data(), f->seg_start, 4 * (f->nseg + 1), cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        f->nvrows = nv;
        GBK_CUDA(cudaMalloc(&f->vrow, 4 * std::max<int64_t>(nv, 1)));
        k_ss_vrows<<<blocks(nnz), 256, 0, s>>>(keys2, flag, vid, nnz, f->vrow, f->chunk_vr);
        GBK_LAUNCHED();
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(stmp);
        cudaFree(tmp);
        cudaFree(keys);
        cudaFree(keys2);
        cudaFree(pos);
        cudaFree(pos2);
        cudaFree(flag);
        cudaFree(vid);
    } else {
        GBK_CUDA(cudaMalloc(&f->vrow, 4));
    }
    // segments without entries start where the next one does
    ss[f->nseg] = (int32_t)nnz;
    for (int32_t g = f->nseg - 1; g >= 0; --g)
        if (ss[g] < 0) ss[g] = ss[g + 1];
    GBK_CUDA(cudaMemcpyAsync(f->seg_start, ss.data(), 4 * (f->nseg + 1), cudaMemcpyHostToDevice, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    *out = f;
    return GBK_SUCCESS;
}

template <int SR, typename T>
int run_impl(const SegSmem* f, int accum, const T* x, T* y, cudaStream_t s) {
    using S = Semiring<SR, T>;
    T* out = accum == GBK_OP_SECOND ? y : (T*)f->tmp;
    if (f->nrows > 0) {
        k_ss_init<T><<<blocks(f->nrows), 256, 0, s>>>(out, f->nrows, S::identity());
        GBK_LAUNCHED();
    }
    if (f->nnz > 0) {
        static bool attr = false;  // one per instantiation
        if (!attr) {
            GBK_CUDA(cudaFuncSetAttribute(k_segsmem<SR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(kSegCols * sizeof(T))));
            attr = true;
        }
        k_segsmem<SR, T><<<(unsigned)num_sms(), kSegThreads, kSegCols * sizeof(T), s>>>(
            f->col, (const T*)f->val, f->head, f->chunk_vr, f->vrow, f->seg_start, f->nseg, f->nnz, f->ncols,
            f->nvrows, f->nrows, x, out, f->err);
        GBK_LAUNCHED();
        if (f->check) {  // first call on this structure: confirm no index check fired
            int32_t e = 0;
            GBK_CUDA(cudaMemcpyAsync(&e, f->err, 4, cudaMemcpyDeviceToHost, s));
            GBK_CUDA(cudaStreamSynchronize(s));
            GBK_REQUIRE(e == 0, GBK_PANIC, "staged CSR_SEG: index check %d failed", e);
            const_cast<SegSmem*>(f)->check = false;
        }
    }
    if (accum != GBK_OP_SECOND && f->nrows > 0) {
        k_ss_accum<T><<<blocks(f->nrows), 256, 0, s>>>(y, (const T*)f->tmp, f->nrows, accum);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

template <typename T>
int run_typed(const SegSmem* f, int sr, int accum, const T* x, T* y, cudaStream_t s) {
    switch (sr) {
#define SS_CASE(SRV) \
    case SRV: return run_impl<SRV, T>(f, accum, x, y, s);
        SS_CASE(GBK_PLUS_TIMES)
        SS_CASE(GBK_PLUS_SECOND)
        SS_CASE(GBK_PLUS_ONE)
        SS_CASE(GBK_MIN_PLUS)
        SS_CASE(GBK_MIN_SECOND)
        SS_CASE(GBK_FIRST_MIN)
        SS_CASE(GBK_MIN_NOTEQ)
        SS_CASE(GBK_LOR_LAND)
        SS_CASE(GBK_STRUCTURAL_BOOL)
#undef SS_CASE
        default: return GBK_UNSUPPORTED;
    }
}

}  // namespace

int build_segsmem(const CsrView& a, int dtype, SegSmem** out, cudaStream_t s) {
    GBK_REQUIRE(a.ncols <= (int64_t)kSegCols * 65536, GBK_UNSUPPORTED, "staged CSR_SEG: too many columns");
    return dtype == GBK_F32 ? build_impl<float>(a, out, s) : build_impl<int32_t>(a, out, s);
}

int run_segsmem(const SegSmem* f, int sr, int accum, int dtype, const void* x, void* y, cudaStream_t s) {
    if (dtype == GBK_F32) return run_typed<float>(f, sr, accum, (const float*)x, (float*)y, s);
    if (dtype == GBK_I32) return run_typed<int32_t>(f, sr, accum, (const int32_t*)x, (int32_t*)y, s);
    return GBK_UNSUPPORTED;
}

void free_segsmem(SegSmem* f) {
    if (!f) return;
    cudaFree(f->col);
    cudaFree(f->val);
    cudaFree(f->head);
    cudaFree(f->chunk_vr);
    cudaFree(f->vrow);
    cudaFree(f->seg_start);
    cudaFree(f->tmp);
    cudaFree(f->err);
    delete f;
}

size_t segsmem_bytes(const SegSmem* f) {
    if (!f) return 0;
    return (size_t)f->nnz * 6 + (size_t)(f->nnz / 32 + 2) * 8 + (size_t)f->nvrows * 4 + (size_t)(f->nseg + 1) * 4 +
           (size_t)f->nrows * 4;
}

}  // namespace gbk
