// Masked SpGEMM C<M> = A (+.x) B by sorted-list intersection.
//
// Replaces SpMSpM_masked_ikj (src/backend/spmspm/spmspm_masked_hash_based_gustavson.h:9-168),
// which builds a hash set per mask row and a hash map of partial sums.  On
// the GPU every stored (i, j) of the mask is one intersection of row i of A
// with column j of B (both sorted): a warp takes 32 consecutive mask
// entries and, entry by entry, its lanes split the shorter list and binary
// search each element in the longer one, so a hub pair is spread over the
// warp and light pairs cost a few instructions each.
//
// Unmasked SpGEMM C = A (+.x) B replaces SpMSpM_unmasked_ikj
// (src/backend/spmspm/spmspm_hash_based_gustavson.h:9-148, a hash map per
// row of C) by expand-sort-compress in row blocks: every product
// A_ik * B_kj is written with its (i, j) key (one thread per product, found
// by binary search over the per-entry product offsets), the block is radix
// sorted by key, equal keys are reduced with the semiring's add, and sums
// equal to 0 are dropped as the reference keeps only val != 0.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <vector>

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

// ---------------------------------------------------------------------------
// unmasked SpGEMM

// products of A's entry e: the degree of row aidx[e] of B
__global__ void k_entry_products(const int32_t* __restrict__ aidx, int64_t nnz, const int32_t* __restrict__ bptr,
                                 int64_t* __restrict__ cnt) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nnz) cnt[e] = bptr[aidx[e] + 1] - bptr[aidx[e]];
}

// product offset of each row's first entry
__global__ void k_row_offsets(const int32_t* __restrict__ aptr, int64_t nrows, const int64_t* __restrict__ off,
                              int64_t* __restrict__ roff) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r <= nrows) roff[r] = off[aptr[r]];
}

// row of A's entry e
__global__ void k_entry_rows(const int32_t* __restrict__ aptr, int64_t nrows, int64_t nnz, int32_t* __restrict__ arow) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int64_t lo = 0, hi = nrows;  // last row starting at or before e
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (aptr[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    arow[e] = (int32_t)lo;
}

// Products [p0, p1) of the entries [e0, e1) (off: exclusive product offsets
// per entry, off[e1] = p1): key ((row - row0) << colbits | column), value
// mul(a, b); the short keys keep the radix sort to the bits in use.
template <int SR, typename T>
__global__ void k_expand(const int64_t* __restrict__ off, int64_t e0, int64_t e1, int64_t p0, int64_t p1,
                         const int32_t* __restrict__ arow, int32_t row0, int colbits, const int32_t* __restrict__ aidx,
                         const T* __restrict__ aval,
                         const int32_t* __restrict__ bptr, const int32_t* __restrict__ bidx,
                         const T* __restrict__ bval, unsigned long long* __restrict__ key, T* __restrict__ val) {
    using S = Semiring<SR, T>;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < p1; p += stride) {
        int64_t lo = e0, hi = e1;  // last entry whose products start at or before p
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (off[mid] <= p)
                lo = mid;
            else
                hi = mid;
        }
        const int32_t k = aidx[lo];
        const int64_t f = bptr[k] + (p - off[lo]);
        key[p - p0] = ((unsigned long long)(uint32_t)(arow[lo] - row0) << colbits) | (unsigned long long)(uint32_t)bidx[f];
        val[p - p0] = S::mul(aval[lo], bval[f]);
    }
}

template <int SR, typename T>
struct SemiringAdd {
    __device__ __forceinline__ T operator()(const T& a, const T& b) const { return Semiring<SR, T>::add(a, b); }
};

template <typename T>
struct NonZero {
    __device__ __forceinline__ bool operator()(const T& v) const { return v != T(0); }
};

__global__ void k_split_keys(const unsigned long long* __restrict__ key, int64_t n, int32_t row0, int colbits,
                             int32_t* __restrict__ row, int32_t* __restrict__ col) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    row[i] = row0 + (int32_t)(key[i] >> colbits);
    col[i] = (int32_t)(key[i] & ((1ull << colbits) - 1));
}

// ptr[r] = first entry of row >= r (rows ascending)
__global__ void k_bounds(const int32_t* __restrict__ row, int64_t nnz, int64_t nrows, int32_t* __restrict__ ptr) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nnz) return;
    const int64_t lo = i == 0 ? 0 : (int64_t)row[i - 1] + 1;
    const int64_t hi = i == nnz ? nrows : (int64_t)row[i];
    for (int64_t r = lo; r <= hi; ++r) ptr[r] = (int32_t)i;
}

template <typename T>
__global__ void k_nonzero_flags(const T* __restrict__ v, int64_t n, uint8_t* __restrict__ flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = v[i] != T(0);
}

unsigned nb(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

// Device scratch from the stream-ordered pool (reused across calls), freed
// on the stream on every exit.
struct Scratch {
    cudaStream_t s;
    std::vector<void*> p;
    explicit Scratch(cudaStream_t st) : s(st) {}
    ~Scratch() {
        for (void* q : p) cudaFreeAsync(q, s);
    }
    template <typename X>
    int get(X** x, size_t bytes) {
        void* q = nullptr;
        if (cudaMallocAsync(&q, std::max<size_t>(bytes, 16), s) != cudaSuccess) return GBK_OUT_OF_MEMORY;
        p.push_back(q);
        *x = (X*)q;
        return GBK_SUCCESS;
    }
};

// Products per block: keys, values and their sorted copies, about 24 bytes
// each.  GBK_MXM_BLOCK_PRODUCTS (at least 1) overrides it, so small products
// can exercise several blocks.
constexpr int64_t kBlockProductsDefault = 64ll << 20;

int64_t block_products() {
    const char* e = getenv("GBK_MXM_BLOCK_PRODUCTS");
    const long long v = e ? atoll(e) : 0;
    return v >= 1 ? (int64_t)v : kBlockProductsDefault;
}

template <int SR, typename T>
int mxm_unmasked(gbk_matrix* out, const CsrView& a, const CsrView& b, cudaStream_t s) {
    const int64_t n = a.nrows, m = b.ncols, annz = a.nnz;
    Scratch dev(s);
    auto need = [&](int rc) { return rc == GBK_SUCCESS; };
    int64_t* off = nullptr;
    int32_t* arow = nullptr;
    if (!need(dev.get(&off, 8 * (annz + 1))) || !need(dev.get(&arow, 4 * annz))) {
        set_error("gbk_mxm: out of device memory");
        return GBK_OUT_OF_MEMORY;
    }
    if (annz > 0) {
        k_entry_products<<<nb(annz), 256, 0, s>>>(a.idx, annz, b.ptr, off);
        GBK_LAUNCHED();
        k_entry_rows<<<nb(annz), 256, 0, s>>>(a.ptr, n, annz, arow);
        GBK_LAUNCHED();
    }
    GBK_CUDA(cudaMemsetAsync(off + annz, 0, 8, s));
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, off, off, annz + 1, s);
        void* tmp = nullptr;
        if (!need(dev.get(&tmp, tb))) return GBK_OUT_OF_MEMORY;
        GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, off, off, annz + 1, s));
        count_launch(1);
    }
    // product offsets at row starts, on the host, to cut row blocks
    int64_t* roff = nullptr;
    if (!need(dev.get(&roff, 8 * (n + 1)))) return GBK_OUT_OF_MEMORY;
    k_row_offsets<<<nb(n + 1), 256, 0, s>>>(a.ptr, n, off, roff);
    GBK_LAUNCHED();
    std::vector<int32_t> hptr(n + 1);
    std::vector<int64_t> hroff(n + 1);
    GBK_CUDA(cudaMemcpyAsync(hptr.data(), a.ptr, 4 * (n + 1), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaMemcpyAsync(hroff.data(), roff, 8 * (n + 1), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    // blocks of whole rows with at most kBlockProducts products (a single row may exceed it)
    std::vector<int64_t> cuts{0};
    const int64_t kBlockProducts = block_products();
    {
        int64_t r = 0;
        while (r < n) {
            const int64_t base = hroff[r];
            int64_t r1 = r + 1;
            int64_t lo = r + 1, hi = n;  // furthest row end within the budget
            while (lo <= hi) {
                const int64_t mid = (lo + hi) / 2;
                if (hroff[mid] - base <= kBlockProducts) {
                    r1 = mid;
                    lo = mid + 1;
                } else {
                    hi = mid - 1;
                }
            }
            cuts.push_back(r1);
            r = r1;
        }
    }
    int64_t maxp = 0;
    for (size_t c = 0; c + 1 < cuts.size(); ++c)
        maxp = std::max<int64_t>(maxp, hroff[cuts[c + 1]] - hroff[cuts[c]]);
    unsigned long long *key = nullptr, *key2 = nullptr;
    T *val = nullptr, *val2 = nullptr;
    int64_t* nsel = nullptr;
    if (!need(dev.get(&key, 8 * maxp)) || !need(dev.get(&key2, 8 * maxp)) || !need(dev.get(&val, sizeof(T) * maxp)) ||
        !need(dev.get(&val2, sizeof(T) * maxp)) || !need(dev.get(&nsel, 16))) {
        set_error("gbk_mxm: out of device memory for %lld products per block", (long long)maxp);
        return GBK_OUT_OF_MEMORY;
    }
    // scratch sized for the largest block
    size_t t_sort = 0, t_red = 0, t_sel = 0;
    int rowbits = 1;
    while ((1ll << rowbits) < n) ++rowbits;
    int colbits = 1;
    while ((1ll << colbits) < m) ++colbits;
    cub::DeviceRadixSort::SortPairs(nullptr, t_sort, key, key2, val, val2, maxp, 0, rowbits + colbits, s);
    cub::DeviceReduce::ReduceByKey(nullptr, t_red, key2, key, val2, val, nsel, SemiringAdd<SR, T>(), maxp, s);
    uint8_t* flag = nullptr;
    if (!need(dev.get(&flag, maxp))) return GBK_OUT_OF_MEMORY;
    cub::DeviceSelect::Flagged(nullptr, t_sel, key, flag, key2, nsel + 1, maxp, s);
    size_t t_if = 0;
    cub::DeviceSelect::If(nullptr, t_if, val, val2, nsel, maxp, NonZero<T>(), s);
    void* tmp = nullptr;
    const size_t tbytes = std::max(std::max(t_sort, t_red), std::max(t_sel, t_if)) + 256;
    if (!need(dev.get(&tmp, tbytes))) return GBK_OUT_OF_MEMORY;
    // per block: expand, sort, reduce, drop zeros; the kept entries are appended
    std::vector<unsigned long long*> okeys;
    std::vector<T*> ovals;
    std::vector<int64_t> ocnt;
    std::vector<int64_t> orow0;  // first row of each kept block
    int64_t total = 0;
    for (size_t c = 0; c + 1 < cuts.size(); ++c) {
        const int64_t e0 = hptr[cuts[c]], e1 = hptr[cuts[c + 1]];
        const int64_t p0 = hroff[cuts[c]], p1 = hroff[cuts[c + 1]], np = p1 - p0;
        if (np == 0) continue;
        const unsigned grid = (unsigned)std::min<int64_t>(nb(np), (int64_t)num_sms() * 32);
        k_expand<SR, T><<<grid, 256, 0, s>>>(off, e0, e1, p0, p1, arow, (int32_t)cuts[c], colbits, a.idx,
                                             (const T*)a.val, b.ptr, b.idx, (const T*)b.val, key, val);
        GBK_LAUNCHED();
        int brows = 1;  // bits of the block's row span
        while ((1ll << brows) < cuts[c + 1] - cuts[c]) ++brows;
        size_t tb = tbytes;
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, val, val2, np, 0, brows + colbits, s));
        tb = tbytes;
        GBK_CUDA(cub::DeviceReduce::ReduceByKey(tmp, tb, key2, key, val2, val, nsel, SemiringAdd<SR, T>(), np, s));
        count_launch(2);
        int64_t nu = 0;
        GBK_CUDA(cudaMemcpyAsync(&nu, nsel, 8, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        // drop the zero sums (keys and values compacted by the same flags)
        {
            unsigned long long* kk = nullptr;
            T* vv = nullptr;
            if (!need(dev.get(&kk, 8 * std::max<int64_t>(nu, 1))) || !need(dev.get(&vv, sizeof(T) * std::max<int64_t>(nu, 1)))) {
                set_error("gbk_mxm: out of device memory for a block's result");
                return GBK_OUT_OF_MEMORY;
            }
            okeys.push_back(kk);
            ovals.push_back(vv);
            orow0.push_back(cuts[c]);
            tb = tbytes;
            GBK_CUDA(cub::DeviceSelect::If(tmp, tb, val, vv, nsel, nu, NonZero<T>(), s));
            count_launch(1);
            // the same selection for the keys: flags from the values
            k_nonzero_flags<T><<<nb(nu), 256, 0, s>>>(val, nu, flag);
            GBK_LAUNCHED();
            tb = tbytes;
            GBK_CUDA(cub::DeviceSelect::Flagged(tmp, tb, key, flag, kk, nsel + 1, nu, s));
            count_launch(1);
            int64_t kept[2] = {0, 0};
            GBK_CUDA(cudaMemcpyAsync(kept, nsel, 16, cudaMemcpyDeviceToHost, s));
            GBK_CUDA(cudaStreamSynchronize(s));
            ocnt.push_back(kept[0]);
            total += kept[0];
        }
    }
    GBK_REQUIRE(total < INT32_MAX, GBK_INVALID_VALUE, "gbk_mxm: the product has %lld entries (int32 limit)",
                (long long)total);
    // CSR of the result
    int32_t *row = nullptr, *col = nullptr, *ptr = nullptr;
    T* cval = nullptr;
    if (!need(dev.get(&row, 4 * total)) || !need(dev.get(&col, 4 * total)) || !need(dev.get(&ptr, 4 * (n + 1))) ||
        !need(dev.get(&cval, sizeof(T) * total))) {
        set_error("gbk_mxm: out of device memory for the result");
        return GBK_OUT_OF_MEMORY;
    }
    int64_t at = 0;
    for (size_t c = 0; c < okeys.size(); ++c) {
        if (ocnt[c] > 0) {
            k_split_keys<<<nb(ocnt[c]), 256, 0, s>>>(okeys[c], ocnt[c], (int32_t)orow0[c], colbits, row + at, col + at);
            GBK_LAUNCHED();
            GBK_CUDA(cudaMemcpyAsync(cval + at, ovals[c], sizeof(T) * ocnt[c], cudaMemcpyDeviceToDevice, s));
        }
        at += ocnt[c];
    }
    k_bounds<<<nb(total + 1), 256, 0, s>>>(row, total, n, ptr);
    GBK_LAUNCHED();
    GBK_CUDA(cudaStreamSynchronize(s));
    return gbk_matrix_create_csr(out, n, m, total, ptr, col, cval, std::is_same<T, float>::value ? GBK_F32 : GBK_I32,
                                 1, s);
}

// ---------------------------------------------------------------------------
// triangle counting

// 1 where A and its CSC differ (A not symmetric) or a diagonal entry exists
__global__ void k_sym_loop_check(const int32_t* __restrict__ ap, const int32_t* __restrict__ ai,
                                 const int32_t* __restrict__ tp, const int32_t* __restrict__ ti, int64_t n,
                                 int64_t nnz, int* __restrict__ bad) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e <= n && ap[e] != tp[e]) atomicOr(bad, 1);
    if (e < nnz && ai[e] != ti[e]) atomicOr(bad, 1);
    if (e < n) {
        for (int32_t k = ap[e]; k < ap[e + 1]; ++k)
            if (ai[k] == (int32_t)e) atomicOr(bad, 2);
    }
}

// keep edge (u, v) when (deg u, u) < (deg v, v): each undirected edge once,
// from its lower-degree end
__device__ __forceinline__ bool oriented(const int32_t* ap, int32_t u, int32_t v) {
    const int32_t du = ap[u + 1] - ap[u], dv = ap[v + 1] - ap[v];
    return du < dv || (du == dv && u < v);
}

__global__ void k_orient_counts(const int32_t* __restrict__ ap, const int32_t* __restrict__ ai, int64_t n,
                                int32_t* __restrict__ cnt) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    int32_t c = 0;
    for (int32_t k = ap[u]; k < ap[u + 1]; ++k) c += oriented(ap, (int32_t)u, ai[k]);
    cnt[u] = c;
}

__global__ void k_orient_fill(const int32_t* __restrict__ ap, const int32_t* __restrict__ ai, int64_t n,
                              const int32_t* __restrict__ op, int32_t* __restrict__ oi, int32_t* __restrict__ orow) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    int32_t w = op[u];
    for (int32_t k = ap[u]; k < ap[u + 1]; ++k)
        if (oriented(ap, (int32_t)u, ai[k])) {
            oi[w] = ai[k];
            orow[w] = (int32_t)u;
            ++w;
        }
}

// Sum over oriented edges (u, v) of |N+(u) ∩ N+(v)| (rows sorted by id): a
// warp per edge, lanes walk the shorter list and binary-search the longer.
__global__ void k_oriented_triangles(const int32_t* __restrict__ op, const int32_t* __restrict__ oi,
                                     const int32_t* __restrict__ orow, int64_t m,
                                     unsigned long long* __restrict__ total) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long mine = 0;
    for (int64_t e = warp; e < m; e += nwarps) {
        const int32_t u = orow[e], v = oi[e];
        const int32_t u0 = op[u], u1 = op[u + 1], v0 = op[v], v1 = op[v + 1];
        const bool us = (u1 - u0) <= (v1 - v0);
        const int32_t s0 = us ? u0 : v0, s1 = us ? u1 : v1, l0 = us ? v0 : u0, l1 = us ? v1 : u1;
        for (int32_t p = s0 + lane; p < s1; p += 32) {
            const int32_t key = oi[p];
            int32_t lo = l0, hi = l1;
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (oi[mid] < key)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            mine += (lo < l1 && oi[lo] == key);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, off);
    if (lane == 0 && mine) atomicAdd(total, mine);
}

}  // namespace

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_triangle_count(gbk_matrix A, uint64_t* count, void* stream) {
    GBK_REQUIRE(A && count, GBK_NULL_POINTER, "gbk_triangle_count: NULL argument");
    GBK_REQUIRE(A->csr.nrows == A->csr.ncols, GBK_DIMENSION_MISMATCH, "gbk_triangle_count: A is not square");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ensure_csc(A, s);
    if (rc) return rc;
    const CsrView& a = A->csr;
    const CsrView& t = A->csc;
    const int64_t n = a.nrows, nnz = a.nnz;
    Scratch dev(s);
    int* bad = nullptr;
    unsigned long long* total = nullptr;
    if (dev.get(&bad, 4) || dev.get(&total, 8)) return GBK_OUT_OF_MEMORY;
    GBK_CUDA(cudaMemsetAsync(bad, 0, 4, s));
    GBK_CUDA(cudaMemsetAsync(total, 0, 8, s));
    k_sym_loop_check<<<nb(std::max<int64_t>(n + 1, nnz)), 256, 0, s>>>(a.ptr, a.idx, t.ptr, t.idx, n, nnz, bad);
    GBK_LAUNCHED();
    int hbad = 0;
    GBK_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    if (hbad) {
        // not a simple undirected graph: Burkhardt's sum (sum ((A * A) .* A)) / 6 as it stands
        gbk_matrix C = nullptr;
        rc = gbk_mxm_masked(&C, A, A, A, GBK_PLUS_ONE, GBK_I32, stream);
        if (rc) return rc;
        const CsrView& c = C->csr;
        void* tmp = nullptr;
        size_t tb = 0;
        long long* sum = nullptr;
        rc = dev.get(&sum, 8);
        if (!rc) {
            cub::DeviceReduce::Sum(nullptr, tb, (const int32_t*)c.val, sum, c.nnz, s);
            rc = dev.get(&tmp, tb);
        }
        long long hs = 0;
        if (!rc && cub::DeviceReduce::Sum(tmp, tb, (const int32_t*)c.val, sum, c.nnz, s) == cudaSuccess &&
            cudaMemcpyAsync(&hs, sum, 8, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
            cudaStreamSynchronize(s) == cudaSuccess) {
            count_launch(1);
            *count = (uint64_t)(hs / 6);
        } else if (!rc) {
            rc = cuda_fail(cudaGetLastError(), "triangle count reduce", __FILE__, __LINE__);
        }
        gbk_matrix_destroy(C);
        return rc;
    }
    // symmetric, no self loops: orient by (degree, id) and count each triangle once
    int32_t *cnt = nullptr, *op = nullptr, *oi = nullptr, *orow = nullptr;
    if (dev.get(&cnt, 4 * (n + 1)) || dev.get(&op, 4 * (n + 1))) return GBK_OUT_OF_MEMORY;
    k_orient_counts<<<nb(n), 256, 0, s>>>(a.ptr, a.idx, n, cnt);
    GBK_LAUNCHED();
    GBK_CUDA(cudaMemsetAsync(cnt + n, 0, 4, s));
    {
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, op, n + 1, s);
        void* tmp = nullptr;
        if (dev.get(&tmp, tb)) return GBK_OUT_OF_MEMORY;
        GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, op, n + 1, s));
        count_launch(1);
    }
    int32_t m = 0;
    GBK_CUDA(cudaMemcpyAsync(&m, op + n, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    if (dev.get(&oi, 4 * (int64_t)m) || dev.get(&orow, 4 * (int64_t)m)) return GBK_OUT_OF_MEMORY;
    k_orient_fill<<<nb(n), 256, 0, s>>>(a.ptr, a.idx, n, op, oi, orow);
    GBK_LAUNCHED();
    if (m > 0) {
        const int64_t warps = std::min<int64_t>(m, (int64_t)num_sms() * 64);
        k_oriented_triangles<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(op, oi, orow, m, total);
        GBK_LAUNCHED();
    }
    unsigned long long ht = 0;
    GBK_CUDA(cudaMemcpyAsync(&ht, total, 8, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    *count = (uint64_t)ht;
    return GBK_SUCCESS;
}

extern "C" int gbk_mxm(gbk_matrix* out, gbk_matrix A, gbk_matrix B, gbk_semiring sr, void* stream) {
    GBK_REQUIRE(out && A && B, GBK_NULL_POINTER, "gbk_mxm: NULL argument");
    GBK_REQUIRE(A->vtype == B->vtype, GBK_DOMAIN_MISMATCH, "gbk_mxm: A and B value types differ");
    GBK_REQUIRE(A->csr.ncols == B->csr.nrows, GBK_DIMENSION_MISMATCH, "gbk_mxm: A is %lldx%lld, B %lldx%lld",
                (long long)A->csr.nrows, (long long)A->csr.ncols, (long long)B->csr.nrows, (long long)B->csr.ncols);
    cudaStream_t s = (cudaStream_t)stream;
#define MXM_CASE(SRV)                                                                                 \
    case SRV:                                                                                         \
        return A->vtype == GBK_F32 ? mxm_unmasked<SRV, float>(out, A->csr, B->csr, s)                 \
                                   : mxm_unmasked<SRV, int32_t>(out, A->csr, B->csr, s);
    switch (sr) {
        MXM_CASE(GBK_PLUS_TIMES)
        MXM_CASE(GBK_PLUS_SECOND)
        MXM_CASE(GBK_PLUS_ONE)
        MXM_CASE(GBK_MIN_PLUS)
        MXM_CASE(GBK_MIN_SECOND)
        MXM_CASE(GBK_LOR_LAND)
        default:
            set_error("gbk_mxm: semiring %d not provided (plus-times, plus-second, plus-one, min-plus, "
                      "min-second, or-and)",
                      (int)sr);
            return GBK_UNSUPPORTED;
    }
#undef MXM_CASE
}

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
    void* vals = nullptr;  // from the stream-ordered pool: results of this size recur (triangle counting)
    GBK_CUDA(cudaMallocAsync(&vals, 4 * (m.nnz > 0 ? m.nnz : 1), s));
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
    cudaFreeAsync(vals, s);
    return rc;
}
