// SELL-C-sigma with the x window staged in shared memory.
//
// The reference's SELL-C-sigma (src/backend/matrix/containers/sell_c/
// build.hpp:27-295, src/backend/spmv/spmv_sell_c.h:14-170) sorts rows by
// length inside sigma-row windows, packs C rows per chunk column-major and
// gathers x per entry.  On B200 those gathers are bound by the L1 gather rate
// (one sector per lane), so here the columns are also cut into windows of
// kSwCols columns (192 KiB of 4-byte x, one shared-memory copy per CTA), the
// SELL-C-sigma layout is built inside every window, and x comes from shared
// memory:
//   * optionally the columns are renumbered by in-degree first (the order of
//     the reference's LAV format), which packs the most used columns into the
//     first windows;
//   * the entries of one row inside one window form a virtual row; virtual
//     rows longer than kSwPiece entries are cut into pieces of kSwPiece;
//   * inside each window the pieces are sorted by length, descending
//     (sigma = the whole window; ties in row order), and every 32 consecutive
//     pieces form a slice (C = 32, one slice per warp step);
//   * a slice of L steps stores L x 32 entries column-major -- entry k of the
//     piece in lane l at slice offset + 32 k + l -- as a 16-bit window position
//     (bank-swizzled) and the value; each lane knows its piece's output row
//     and length;
//   * work items: a slice of more than kSwShort steps alone, or a run of up to
//     8 consecutive short slices of at most 8 steps in all (their entries are
//     contiguous, so one round of loads fetches the whole run);
//   * 148 persistent CTAs (one per SM, 1024 threads) take shares of whole work
//     items, cut by a cost model and then calibrated from timed launches; for
//     every window in its share a CTA copies the x window into shared memory
//     once; its warps take items from a shared counter, the next item's
//     descriptor loaded while one runs; a lane sums its piece and folds the sum
//     into y with one atomic of the semiring's add.
// Float sums therefore add pieces in an order that varies between runs
// (within the FP32 tolerance); integer, min and or results are exact.
// Semirings whose add is not associative fall back to the CSR kernels.
#include <algorithm>
#include <type_traits>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace gbk {

constexpr int kSwCols = 49152;     // x values per window (192 KiB of 4-byte values)
constexpr int kSwThreads = 1024;
constexpr int kSwPiece = 32;       // longest piece of a virtual row: a slice is at most 32 steps, so no
                                   // warp holds its CTA at a window change for long (< 512: 9-bit sort key)
constexpr int kSwUnroll = 8;       // steps of a long slice whose loads are in flight together
constexpr int kSwShort = 8;        // slices of at most this many steps are grouped into work items
constexpr size_t kSwSmemBytes = 4 * (size_t)kSwCols;

// Window position of column c: the column's bank bits XOR three higher
// 5-bit groups (a permutation inside each 32-column block), so columns whose
// low bits are zero -- the hubs of power-law graphs -- spread over the banks.
__host__ __device__ __forceinline__ uint32_t sw_pos(uint32_t c) {
    return c ^ (((c >> 5) ^ (c >> 10) ^ (c >> 15)) & 31u);
}

struct SellW {
    int64_t nrows = 0, ncols = 0, nnz = 0;
    int32_t nwin = 0;
    int64_t nslices = 0, npieces = 0, padded = 0;
    uint16_t* col = nullptr;        // padded entries: sw_pos of the column inside its window
    void* val = nullptr;            // padded entries
    int64_t nitems = 0;
    int4* item = nullptr;           // work items: (first padded entry, first slice, steps of a long slice or the
                                    // 4-bit step counts of a run of short slices, 0 or the run's slices)
    int32_t* prow = nullptr;        // nslices * 32: output row of each lane's piece (-1: empty lane)
    uint16_t* plen = nullptr;       // nslices * 32: entries of each lane's piece
    int32_t* win_item = nullptr;    // nwin + 1: first work item of each window
    int32_t nshares = 0;
    int32_t* share = nullptr;       // nshares + 1 work-item offsets of the CTAs' shares
    int32_t* new_to_old = nullptr;  // columns renumbered by in-degree (NULL: original order)
    void* xr = nullptr;             // x in the renumbered order
    void* tmp = nullptr;            // nrows: the product before the accumulator
    int32_t* err = nullptr;         // first failed index check seen by the kernel (0 = none)
    bool check = true;              // read err back after the first launch
};

namespace {

unsigned sw_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

int sw_scan_excl(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s) {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), s));
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int)n, s));
    count_launch(1);
    GBK_CUDA(cudaFreeAsync(tmp, s));
    return GBK_SUCCESS;
}

// ---- build ------------------------------------------------------------------

// key = (window << 32) | row, value = entry position; one thread per entry,
// its row by binary search in the row pointers (a thread per row would walk
// a hub row of 10^5 entries alone)
__global__ void k_sw_keys(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, int64_t n, int64_t nnz,
                          unsigned long long* __restrict__ keys, int32_t* __restrict__ pos) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int64_t lo = 0, hi = n;  // largest r with ptr[r] <= e
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (ptr[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    keys[e] = ((unsigned long long)(idx[e] / kSwCols) << 32) | (unsigned long long)lo;
    pos[e] = (int32_t)e;
}

// vs[i] = i where a virtual row starts, else 0 (a running max gives each
// entry its virtual row's first entry)
__global__ void k_sw_vstart(const unsigned long long* __restrict__ keys, int64_t nnz, int32_t* __restrict__ vs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nnz) vs[i] = (i == 0 || keys[i] != keys[i - 1]) ? (int32_t)i : 0;
}

// a piece starts every kSwPiece entries of a virtual row
__global__ void k_sw_pflag(const int32_t* __restrict__ vstart, int64_t nnz, int32_t* __restrict__ pflag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nnz) pflag[i] = ((i - vstart[i]) % kSwPiece) == 0;
    if (i == nnz) pflag[i] = 0;
}

__global__ void k_sw_pfirst(const int32_t* __restrict__ pflag, const int32_t* __restrict__ pid, int64_t nnz,
                            int32_t* __restrict__ pfirst) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nnz && pflag[i]) pfirst[pid[i]] = (int32_t)i;
}

// sort key of a piece: window, then length descending (len <= kSwPiece < 512)
__global__ void k_sw_pkey(const int32_t* __restrict__ pfirst, const unsigned long long* __restrict__ keys,
                          int64_t np, uint32_t* __restrict__ pkey, int32_t* __restrict__ pidx) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int32_t len = pfirst[p + 1] - pfirst[p];
    const uint32_t w = (uint32_t)(keys[pfirst[p]] >> 32);
    pkey[p] = (w << 9) | (uint32_t)(511 - len);
    pidx[p] = (int32_t)p;
}

__global__ void k_sw_wcount(const uint32_t* __restrict__ pkey_sorted, int64_t np, int32_t* __restrict__ wcnt) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < np) warp_count(wcnt, (int32_t)(pkey_sorted[j] >> 9));  // sorted: one atomic per window per warp
}

__global__ void k_sw_wslices(const int32_t* __restrict__ wcnt, int32_t nwin, int32_t* __restrict__ wsl) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nwin) wsl[w] = (wcnt[w] + 31) / 32;
    if (w == nwin) wsl[w] = 0;
}

// place every piece in its slice / lane; lane 0 of a slice sets its length
__global__ void k_sw_place(const uint32_t* __restrict__ pkey_sorted, const int32_t* __restrict__ pidx_sorted,
                           int64_t np, const int32_t* __restrict__ wpfirst, const int32_t* __restrict__ win_slice,
                           const int32_t* __restrict__ pfirst, const unsigned long long* __restrict__ keys,
                           int32_t* __restrict__ prow, uint16_t* __restrict__ plen, int32_t* __restrict__ slen,
                           int32_t* __restrict__ pslot) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= np) return;
    const uint32_t w = pkey_sorted[j] >> 9;
    const int32_t len = 511 - (int32_t)(pkey_sorted[j] & 511u);
    const int64_t r = j - wpfirst[w];
    const int64_t slot = ((int64_t)win_slice[w] + r / 32) * 32 + (r & 31);
    const int32_t p = pidx_sorted[j];
    prow[slot] = (int32_t)(keys[pfirst[p]] & 0xffffffffull);
    plen[slot] = (uint16_t)len;
    pslot[p] = (int32_t)slot;
    if ((r & 31) == 0) slen[slot / 32] = len;
}

__global__ void k_sw_steps(const int32_t* __restrict__ slen, int64_t ns, long long* __restrict__ ent) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < ns) ent[s] = 32ll * slen[s];
    if (s == ns) ent[s] = 0;
}

template <typename T>
__global__ void k_sw_fill(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ pos,
                          const int32_t* __restrict__ pflag, const int32_t* __restrict__ pid,
                          const int32_t* __restrict__ pfirst, const int32_t* __restrict__ pslot,
                          const long long* __restrict__ soff, const int32_t* __restrict__ idx,
                          const T* __restrict__ v, int64_t nnz, uint16_t* __restrict__ col, T* __restrict__ val) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    const int32_t p = pid[i] + pflag[i] - 1;  // the piece holding entry i
    const int64_t k = i - pfirst[p];
    const int64_t slot = pslot[p];
    const int64_t dst = soff[slot / 32] + 32 * k + (slot & 31);
    const int64_t w = (int64_t)(keys[i] >> 32);
    const int32_t e = pos[i];
    col[dst] = (uint16_t)sw_pos((uint32_t)(idx[e] - w * kSwCols));
    val[dst] = v[e];
}

// ---- SpMV ------------------------------------------------------------------

template <int SR>
struct SwAddClass {  // 0 plus, 1 min, 2 or, -1 not folded atomically
    static constexpr int value = (SR == GBK_PLUS_TIMES || SR == GBK_PLUS_SECOND || SR == GBK_PLUS_ONE) ? 0
                                 : (SR == GBK_MIN_PLUS || SR == GBK_MIN_SECOND || SR == GBK_FIRST_MIN ||
                                    SR == GBK_MIN_NOTEQ)
                                     ? 1
                                 : (SR == GBK_LOR_LAND || SR == GBK_STRUCTURAL_BOOL) ? 2
                                                                                      : -1;
};

// fold a piece's sum v into out[r] with the semiring's add (the add's
// identity never changes y, so it costs no atomic)
template <int SR, typename T>
__device__ __forceinline__ void sw_fold(T* out, int32_t r, T v) {
    using S = Semiring<SR, T>;
    constexpr int cls = SwAddClass<SR>::value;
    if constexpr (cls == 0) {
        if (v != T(0)) atomic_add_any(out + r, v);
    } else if constexpr (cls == 1) {
        if (v < S::identity()) atomic_min_any(out + r, v);
    } else {
        if (v != T(0)) out[r] = T(1);
    }
}

// Copy w values of x into their swizzled shared-memory positions with 4-byte
// asynchronous copies; returns once this thread's copies have landed (the
// caller's barrier publishes them).
template <typename T>
__device__ __forceinline__ void sw_stage(T* xs, const T* src, int w) {
    static_assert(sizeof(T) == 4, "4-byte values");
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(xs);
    for (int i = threadIdx.x; i < w; i += blockDim.x)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst + 4u * sw_pos((uint32_t)i)), "l"(src + i)
                     : "memory");
    asm volatile("cp.async.wait_all;" ::: "memory");
}

template <typename T> __device__ __forceinline__ T sw_ld(const T* p);
// The matrix streams through once per SpMV: last-use loads (measured 1 %
// faster than evict-first ones here, 12 % faster than read-only-cache ones).
template <> __device__ __forceinline__ float sw_ld<float>(const float* p) { return __ldlu(p); }
template <> __device__ __forceinline__ int32_t sw_ld<int32_t>(const int32_t* p) { return __ldlu(p); }

// Fold lane's piece sum into its row (row checked; an empty lane folds nothing).
template <int SR, typename T>
__device__ __forceinline__ void sw_emit(T* out, int32_t r, int32_t ln, T acc, int64_t nrows, bool& bad_row) {
    if (ln <= 0) return;
    if ((uint64_t)(uint32_t)r < (uint64_t)nrows)
        sw_fold<SR, T>(out, r, acc);
    else
        bad_row = true;
}

// One warp's work items of the window part [a, b), taken one at a time from
// the CTA's counter (the next item's descriptor loaded while this one runs).
// An item is either one slice of more than kSwShort steps -- summed 8 steps
// at a time with the next 8 steps' loads already in flight -- or a run of up
// to 8 consecutive short slices of at most 8 steps in all, whose entries,
// rows and lengths all go out in one round of loads.  Index checks: a
// window position past the staged window or a row out of range sets a flag
// (reported once) and the access is clamped or skipped.
template <int SR, typename T>
__device__ __forceinline__ void sw_warp(const uint16_t* __restrict__ col, const T* __restrict__ val,
                                        const int4* __restrict__ item, const int32_t* __restrict__ prow,
                                        const uint16_t* __restrict__ plen, const T* xs, uint32_t wl, int32_t a,
                                        int32_t b, int* next, T* out, int64_t nrows, bool& bad_col, bool& bad_row) {
    using S = Semiring<SR, T>;
    const unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    auto grab = [&]() -> int32_t {
        int t = 0;
        if (lane == 0) t = atomicAdd(next, 1);
        return a + __shfl_sync(kAll, t, 0);
    };
    auto prod = [&](uint32_t c, T v) -> T {
        bad_col |= c > wl;
        return S::mul(v, xs[min(c, wl)]);
    };
    int32_t q = grab();
    if (q >= b) return;
    int4 it = __ldg(item + q);
    for (;;) {
        const int32_t qn = grab();
        int4 itn = make_int4(0, 0, 0, 0);
        if (qn < b) itn = __ldg(item + qn);
        const uint16_t* cp = col + (int64_t)it.x + lane;
        const T* vp = val + (int64_t)it.x + lane;
        if (it.w == 0) {
            // one long slice of it.z steps
            const int L = it.z;
            const int32_t r = __ldg(prow + (int64_t)it.y * 32 + lane);
            const int32_t ln = __ldg(plen + (int64_t)it.y * 32 + lane);
            uint32_t c[kSwUnroll];
            T v[kSwUnroll];
#pragma unroll
            for (int i = 0; i < kSwUnroll; ++i) {  // L > kSwShort >= kSwUnroll: a full first batch
                c[i] = __ldlu(cp + 32 * i);
                v[i] = sw_ld<T>(vp + 32 * i);
            }
            T acc = S::identity();
            int k = 0;
            for (; k + 2 * kSwUnroll <= L; k += kSwUnroll) {
                uint32_t cn[kSwUnroll];
                T vn[kSwUnroll];
#pragma unroll
                for (int i = 0; i < kSwUnroll; ++i) {  // the next batch goes out first
                    cn[i] = __ldlu(cp + 32 * (k + kSwUnroll + i));
                    vn[i] = sw_ld<T>(vp + 32 * (k + kSwUnroll + i));
                }
#pragma unroll
                for (int i = 0; i < kSwUnroll; ++i) {
                    const T p = prod(c[i], v[i]);
                    if (k + i < ln) acc = S::add(acc, p);
                    c[i] = cn[i];
                    v[i] = vn[i];
                }
            }
            // the batch in registers, with the tail's loads (fewer than
            // kSwUnroll steps) issued first as one predicated batch
            const int kt = k + kSwUnroll;
            uint32_t ct[kSwUnroll];
            T vt[kSwUnroll];
#pragma unroll
            for (int i = 0; i < kSwUnroll; ++i) {
                ct[i] = 0;
                vt[i] = T(0);
                if (kt + i < L) {
                    ct[i] = __ldlu(cp + 32 * (kt + i));
                    vt[i] = sw_ld<T>(vp + 32 * (kt + i));
                }
            }
#pragma unroll
            for (int i = 0; i < kSwUnroll; ++i) {
                const T p = prod(c[i], v[i]);
                if (k + i < ln) acc = S::add(acc, p);
            }
#pragma unroll
            for (int i = 0; i < kSwUnroll; ++i) {
                if (kt + i < L) {
                    const T p = prod(ct[i], vt[i]);
                    if (kt + i < ln) acc = S::add(acc, p);
                }
            }
            sw_emit<SR, T>(out, r, ln, acc, nrows, bad_row);
        } else {
            // it.w short slices from slice it.y, lengths in 4-bit fields of it.z
            const int m = it.w;
            int steps = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) steps += j < m ? (it.z >> (4 * j)) & 15 : 0;
            uint32_t c[8];
            T v[8];
            int32_t r[8], ln[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                c[t] = 0;
                v[t] = T(0);
                if (t < steps) {
                    c[t] = __ldlu(cp + 32 * t);
                    v[t] = sw_ld<T>(vp + 32 * t);
                }
            }
            const bool unit = steps == m;  // every slice one step long (the common case)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                r[j] = -1;
                ln[j] = 0;
                if (j < m) {
                    r[j] = __ldg(prow + (int64_t)(it.y + j) * 32 + lane);
                    // a one-step slice's lane holds one entry or none (row -1)
                    if (!unit) ln[j] = __ldg(plen + (int64_t)(it.y + j) * 32 + lane);
                }
            }
            T p[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) p[t] = t < steps ? prod(c[t], v[t]) : S::identity();
            if (unit) {
                // lane's piece j is entry j
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (j < m) sw_emit<SR, T>(out, r[j], r[j] >= 0 ? 1 : 0, p[j], nrows, bad_row);
            } else {
                int base = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (j < m) {
                        const int Lj = (it.z >> (4 * j)) & 15;
                        T acc = S::identity();
#pragma unroll
                        for (int t = 0; t < 8; ++t)
                            if (t >= base && t - base < min(Lj, ln[j])) acc = S::add(acc, p[t]);
                        sw_emit<SR, T>(out, r[j], ln[j], acc, nrows, bad_row);
                        base += Lj;
                    }
                }
            }
        }
        if (qn >= b) break;
        q = qn;
        it = itn;
    }
}

template <int SR, typename T>
__global__ void __launch_bounds__(kSwThreads, 1)
    k_sellw(const uint16_t* __restrict__ col, const T* __restrict__ val, const int4* __restrict__ item,
            const int32_t* __restrict__ prow, const uint16_t* __restrict__ plen, const int32_t* __restrict__ win_item,
            const int32_t* __restrict__ share, int32_t nwin, int64_t ncols, int64_t nrows, const T* __restrict__ x,
            T* out, int32_t* err, long long* clk, int wait_first) {
    extern __shared__ __align__(16) unsigned char sw_smem[];
    T* xs = reinterpret_cast<T*>(sw_smem);
    __shared__ int next_item;
    const long long t0 = clock64();
    // x itself comes from the kernel before this one (renumbered columns): wait
    // for it before staging; with programmatic stream serialisation only the
    // launch overlaps it, otherwise a no-op
    if (wait_first) asm volatile("griddepcontrol.wait;" ::: "memory");
    const int32_t c0 = share[blockIdx.x], c1 = share[blockIdx.x + 1];
    if (c0 >= c1) {  // the whole block leaves together
        if (clk && threadIdx.x == 0) clk[blockIdx.x] = 0;
        return;
    }
    int lo = 0, hi = nwin;  // last window starting at or before c0
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (win_item[mid] <= c0)
            lo = mid;
        else
            hi = mid;
    }
    bool bad_col = false, bad_row = false, waited = false;
    for (int w = lo; w < nwin && win_item[w] < c1; ++w) {
        const int32_t a = max(c0, win_item[w]), b = min(c1, win_item[w + 1]);
        if (a >= b) continue;
        __syncthreads();  // the previous window's readers are done
        if (threadIdx.x == 0) next_item = 0;
        const int64_t col0 = (int64_t)w * kSwCols;
        const int wn = (int)min((int64_t)kSwCols, ncols - col0);
        sw_stage(xs, x + col0, wn);
        __syncthreads();
        if (!waited) {
            // y's initialisation (the kernel before this one on the stream) has
            // finished before the first fold; with programmatic stream
            // serialisation everything above overlaps it, otherwise a no-op
            asm volatile("griddepcontrol.wait;" ::: "memory");
            waited = true;
        }
        const uint32_t wl = (uint32_t)(((wn + 31) & ~31) - 1);  // last staged position
        sw_warp<SR, T>(col, val, item, prow, plen, xs, wl, a, b, &next_item, out, nrows, bad_col, bad_row);
    }
    if (bad_col) atomicCAS(err, 0, 1);
    if (bad_row) atomicCAS(err, 0, 2);
    if (clk) {  // calibration launches: the block's time in SM cycles
        __syncthreads();
        if (threadIdx.x == 0) clk[blockIdx.x] = clock64() - t0;
    }
}

// y = the add's identity and, for renumbered columns, x gathered into the
// new order (one pass for both); lets the SpMV kernel launch early
template <typename T>
__global__ void k_sw_prologue(T* __restrict__ out, int64_t n, T v, const T* __restrict__ x,
                              const int32_t* __restrict__ new_to_old, int64_t nc, T* __restrict__ xr) {
    asm volatile("griddepcontrol.launch_dependents;");
    const int64_t m = new_to_old ? max(n, nc) : n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n) out[i] = v;
        if (new_to_old && i < nc) xr[i] = x[new_to_old[i]];
    }
}

template <typename T>
__global__ void k_sw_accum(T* __restrict__ y, const T* __restrict__ t, int64_t n, int accum) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = binop<T>(accum, y[i], t[i]);
}

template <int SR, typename T>
int launch_sellw(const SellW* f, const T* x, T* out, bool overlap_prev, cudaStream_t s, long long* clk = nullptr,
                 bool wait_first = false) {
    static bool attr = false;  // one per instantiation
    if (!attr) {
        GBK_CUDA(cudaFuncSetAttribute(k_sellw<SR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSwSmemBytes));
        attr = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)f->nshares);
    cfg.blockDim = dim3(kSwThreads);
    cfg.dynamicSmemBytes = kSwSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    la[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = la;
    cfg.numAttrs = overlap_prev ? 1 : 0;
    GBK_CUDA(cudaLaunchKernelEx(&cfg, k_sellw<SR, T>, (const uint16_t*)f->col, (const T*)f->val,
                                (const int4*)f->item, (const int32_t*)f->prow, (const uint16_t*)f->plen,
                                (const int32_t*)f->win_item, (const int32_t*)f->share, f->nwin, f->ncols, f->nrows, x,
                                out, f->err, clk, (int)(wait_first && overlap_prev)));
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

template <int SR, typename T>
int run_impl(const SellW* f, int accum, const T* x, T* y, cudaStream_t s) {
    using S = Semiring<SR, T>;
    const T* xin = f->new_to_old ? (const T*)f->xr : x;
    T* out = accum == GBK_OP_SECOND ? y : (T*)f->tmp;
    const int64_t m = f->new_to_old ? std::max(f->nrows, f->ncols) : f->nrows;
    if (m > 0) {
        const unsigned nb = (unsigned)std::min<int64_t>(sw_blocks(m), 8 * num_sms());
        k_sw_prologue<T><<<nb, 256, 0, s>>>(out, f->nrows, S::identity(), x, f->new_to_old, f->ncols, (T*)f->xr);
        GBK_LAUNCHED();
    }
    if (f->nitems > 0) {
        const int rc = launch_sellw<SR, T>(f, xin, out, m > 0, s, nullptr, f->new_to_old != nullptr);
        if (rc != GBK_SUCCESS) return rc;
        if (f->check) {  // first call on this structure: confirm no index check fired
            int32_t e = 0;
            GBK_CUDA(cudaMemcpyAsync(&e, f->err, 4, cudaMemcpyDeviceToHost, s));
            GBK_CUDA(cudaStreamSynchronize(s));
            GBK_REQUIRE(e == 0, GBK_PANIC, "staged SELL-C: index check %d failed", e);
            const_cast<SellW*>(f)->check = false;
        }
    }
    if (accum != GBK_OP_SECOND && f->nrows > 0) {
        k_sw_accum<T><<<sw_blocks(f->nrows), 256, 0, s>>>(y, (const T*)f->tmp, f->nrows, accum);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

template <typename T>
int run_typed(const SellW* f, int sr, int accum, const T* x, T* y, cudaStream_t s) {
    switch (sr) {
#define SW_CASE(SRV) \
    case SRV: return run_impl<SRV, T>(f, accum, x, y, s);
        SW_CASE(GBK_PLUS_TIMES)
        SW_CASE(GBK_PLUS_SECOND)
        SW_CASE(GBK_PLUS_ONE)
        SW_CASE(GBK_MIN_PLUS)
        SW_CASE(GBK_MIN_SECOND)
        SW_CASE(GBK_FIRST_MIN)
        SW_CASE(GBK_MIN_NOTEQ)
        SW_CASE(GBK_LOR_LAND)
        SW_CASE(GBK_STRUCTURAL_BOOL)
#undef SW_CASE
        default: return GBK_UNSUPPORTED;
    }
}

// Work items from the slices of every window (in window order): a slice of
// more than kSwShort steps alone, else a run of consecutive short slices of
// at most 8 slices and 8 steps in all.
void sw_items(const std::vector<int32_t>& slen, const std::vector<long long>& soff,
              const std::vector<int32_t>& win_slice, std::vector<int4>& items, std::vector<int32_t>& win_item) {
    const int nwin = (int)win_slice.size() - 1;
    items.clear();
    win_item.assign(nwin + 1, 0);
    for (int w = 0; w < nwin; ++w) {
        win_item[w] = (int32_t)items.size();
        int32_t q = win_slice[w];
        const int32_t end = win_slice[w + 1];
        while (q < end) {
            if (slen[q] > kSwShort) {
                items.push_back(make_int4((int32_t)soff[q], q, slen[q], 0));
                ++q;
                continue;
            }
            const int32_t q0 = q;
            int steps = 0, m = 0, packed = 0;
            while (q < end && m < 8 && slen[q] <= kSwShort && steps + slen[q] <= 8) {
                packed |= slen[q] << (4 * m);
                steps += slen[q];
                ++m;
                ++q;
            }
            items.push_back(make_int4((int32_t)soff[q0], q0, packed, m));
        }
    }
    win_item[nwin] = (int32_t)items.size();
}

// Modelled cost of the items before q (acc[q]): an item costs its padded
// entries plus a fixed overhead, a window start the cost of staging it.
std::vector<double> sw_model_cost(const std::vector<int4>& items, const std::vector<int32_t>& win_item) {
    const double kItemCost = 96.0, kWindowCost = 8192.0;
    const int64_t ni = (int64_t)items.size();
    std::vector<double> acc(ni + 1, 0.0);
    size_t w = 0;
    for (int64_t q = 0; q < ni; ++q) {
        int steps = items[q].w == 0 ? items[q].z : 0;
        for (int j = 0; j < items[q].w; ++j) steps += (items[q].z >> (4 * j)) & 15;
        double c = 32.0 * steps + kItemCost;
        while (w + 1 < win_item.size() && win_item[w + 1] <= q) ++w;
        if (win_item[w] == q) c += kWindowCost;
        acc[q + 1] = acc[q] + c;
    }
    return acc;
}

// Cut the items into nsh shares of equal weight (acc: non-decreasing weight
// of the items before q).
void sw_cut_shares(const std::vector<double>& acc, int nsh, std::vector<int32_t>& share) {
    const int64_t ni = (int64_t)acc.size() - 1;
    share.assign(nsh + 1, 0);
    int64_t q = 0;
    for (int b = 1; b < nsh; ++b) {
        const double target = acc[ni] * b / nsh;
        while (q < ni && acc[q] < target) ++q;
        share[b] = (int32_t)q;
    }
    share[nsh] = (int32_t)ni;
}

// Calibrated shares: time every CTA's share (plus-times over x = 1, SM
// cycles, the median of three warm launches), spread each share's time over
// its items by the modelled cost, average with the previous rounds' estimate
// and cut again at equal time; the shares whose slowest CTA was fastest over
// all rounds are kept (the model alone leaves CTAs idle for half of a launch
// on power-law graphs, and a single round's cut moves with timing noise).
constexpr int kSwCalibrationRounds = 12;
constexpr int kSwCalibrationReps = 3;

template <typename T>
__global__ void k_sw_fill_one(T* v, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = T(1);
}

int sw_calibrate(SellW* f, const std::vector<double>& cost, std::vector<int32_t>& share, cudaStream_t s) {
    const int nsh = f->nshares;
    const int64_t ni = (int64_t)cost.size() - 1;
    float* x1 = nullptr;
    long long* clk = nullptr;
    GBK_CUDA(cudaMalloc(&x1, sizeof(float) * std::max<int64_t>(f->ncols, 1)));
    GBK_CUDA(cudaMalloc(&clk, sizeof(long long) * nsh));
    k_sw_fill_one<float><<<sw_blocks(f->ncols), 256, 0, s>>>(x1, f->ncols);
    GBK_LAUNCHED();
    std::vector<long long> t(nsh);
    std::vector<std::vector<long long>> reps(kSwCalibrationReps, std::vector<long long>(nsh));
    std::vector<double> w(ni + 1), wavg;
    std::vector<int32_t> best = share;
    long long best_max = -1;
    int rc = GBK_SUCCESS;
    for (int round = 0; round < kSwCalibrationRounds && rc == GBK_SUCCESS; ++round) {
        rc = launch_sellw<GBK_PLUS_TIMES, float>(f, x1, (float*)f->tmp, false, s, clk);  // warm-up
        for (int rep = 0; rep < kSwCalibrationReps && rc == GBK_SUCCESS; ++rep) {
            rc = launch_sellw<GBK_PLUS_TIMES, float>(f, x1, (float*)f->tmp, false, s, clk);
            if (rc != GBK_SUCCESS) break;
            GBK_CUDA(cudaMemcpyAsync(reps[rep].data(), clk, sizeof(long long) * nsh, cudaMemcpyDeviceToHost, s));
        }
        if (rc != GBK_SUCCESS) break;
        GBK_CUDA(cudaStreamSynchronize(s));
        long long tmax = 0;
        for (int b = 0; b < nsh; ++b) {
            long long v[kSwCalibrationReps];
            for (int r = 0; r < kSwCalibrationReps; ++r) v[r] = reps[r][b];
            std::sort(v, v + kSwCalibrationReps);
            t[b] = v[kSwCalibrationReps / 2];
            tmax = std::max(tmax, t[b]);
        }
        if (best_max < 0 || tmax < best_max) {
            best_max = tmax;
            best = share;
        }
        double tsum = 0, csum = 0;
        for (int b = 0; b < nsh; ++b)
            if (share[b + 1] > share[b] && t[b] > 0) {
                tsum += (double)t[b];
                csum += cost[share[b + 1]] - cost[share[b]];
            }
        if (tsum <= 0 || csum <= 0) break;
        double acc = 0;
        w[0] = 0;
        for (int b = 0; b < nsh; ++b) {
            const int64_t q0 = share[b], q1 = share[b + 1];
            if (q1 <= q0) continue;
            const double cb = cost[q1] - cost[q0];
            const double tb = t[b] > 0 ? (double)t[b] : cb * tsum / csum;
            for (int64_t q = q0 + 1; q <= q1; ++q) w[q] = acc + tb * (cost[q] - cost[q0]) / cb;
            acc += tb;
        }
        if (wavg.empty()) {
            wavg = w;
        } else {
            for (int64_t q = 0; q <= ni; ++q) wavg[q] = 0.5 * (wavg[q] + w[q]);
        }
        sw_cut_shares(wavg, nsh, share);
        GBK_CUDA(cudaMemcpyAsync(f->share, share.data(), 4 * share.size(), cudaMemcpyHostToDevice, s));
    }
    share = best;
    GBK_CUDA(cudaMemcpyAsync(f->share, share.data(), 4 * share.size(), cudaMemcpyHostToDevice, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    cudaFree(x1);
    cudaFree(clk);
    return rc;
}

template <typename T>
int build_impl(const CsrView& a0, bool reorder, SellW** out, cudaStream_t s) {
    SellW* f = new SellW();
    auto fail = [&](int rc) {
        free_sellw(f);
        return rc;
    };
    f->nrows = a0.nrows;
    f->ncols = a0.ncols;
    f->nnz = a0.nnz;
    f->nwin = (int32_t)std::max<int64_t>(1, (a0.ncols + kSwCols - 1) / kSwCols);
    const int64_t nnz = a0.nnz, nc1 = std::max<int64_t>(a0.ncols, 1);
    GBK_CUDA(cudaMalloc(&f->err, 4));
    GBK_CUDA(cudaMemsetAsync(f->err, 0, 4, s));
    GBK_CUDA(cudaMalloc(&f->tmp, sizeof(T) * std::max<int64_t>(a0.nrows, 1)));
    CsrView a = a0;
    int32_t* idx2 = nullptr;
    if (reorder) {
        GBK_CUDA(cudaMalloc(&f->xr, sizeof(T) * nc1));
        int rc = indegree_order(a0, 0.8f, &f->new_to_old, &idx2, nullptr, s);
        if (rc) return fail(rc);
        a.idx = idx2;
    }
    GBK_CUDA(cudaMalloc(&f->win_item, 4 * (f->nwin + 1)));
    if (nnz == 0) {
        GBK_CUDA(cudaMemsetAsync(f->win_item, 0, 4 * (f->nwin + 1), s));
        GBK_CUDA(cudaMalloc(&f->share, 8));
        GBK_CUDA(cudaMemsetAsync(f->share, 0, 8, s));
        f->nshares = 1;
        GBK_CUDA(cudaStreamSynchronize(s));
        cudaFree(idx2);
        *out = f;
        return GBK_SUCCESS;
    }
    unsigned long long *keys = nullptr, *keys2 = nullptr;
    int32_t *pos = nullptr, *pos2 = nullptr, *vs = nullptr, *vstart = nullptr, *pflag = nullptr, *pid = nullptr;
    GBK_CUDA(cudaMallocAsync(&keys, 8 * nnz, s));
    GBK_CUDA(cudaMallocAsync(&keys2, 8 * nnz, s));
    GBK_CUDA(cudaMallocAsync(&pos, 4 * nnz, s));
    GBK_CUDA(cudaMallocAsync(&pos2, 4 * nnz, s));
    GBK_CUDA(cudaMallocAsync(&vs, 4 * nnz, s));
    GBK_CUDA(cudaMallocAsync(&vstart, 4 * nnz, s));
    GBK_CUDA(cudaMallocAsync(&pflag, 4 * (nnz + 1), s));
    GBK_CUDA(cudaMallocAsync(&pid, 4 * (nnz + 1), s));
    // entries by (window, row), in CSR order inside each: the entries come
    // in row order, so a stable sort on the window bits alone is enough
    k_sw_keys<<<sw_blocks(nnz), 256, 0, s>>>(a.ptr, a.idx, a.nrows, nnz, keys, pos);
    GBK_LAUNCHED();
    int win_bits = 1;
    while ((1ll << win_bits) < f->nwin) ++win_bits;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, pos, pos2, (int)nnz, 32, 32 + win_bits, s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), s));
    GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, pos, pos2, (int)nnz, 32, 32 + win_bits, s));
    count_launch(1);
    cudaFreeAsync(tmp, s);
    // pieces: kSwPiece-entry parts of the virtual rows
    k_sw_vstart<<<sw_blocks(nnz), 256, 0, s>>>(keys2, nnz, vs);
    GBK_LAUNCHED();
    size_t mb = 0;
    cub::DeviceScan::InclusiveScan(nullptr, mb, vs, vstart, ::cuda::maximum<int32_t>{}, (int)nnz, s);
    GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(mb, 16), s));
    GBK_CUDA(cub::DeviceScan::InclusiveScan(tmp, mb, vs, vstart, ::cuda::maximum<int32_t>{}, (int)nnz, s));
    count_launch(1);
    cudaFreeAsync(tmp, s);
    k_sw_pflag<<<sw_blocks(nnz + 1), 256, 0, s>>>(vstart, nnz, pflag);
    GBK_LAUNCHED();
    GBK_CUDA(cudaStreamSynchronize(s));
    int rc = sw_scan_excl(pflag, pid, nnz + 1, s);
    if (rc) return fail(rc);
    int32_t np32 = 0;
    GBK_CUDA(cudaMemcpyAsync(&np32, pid + nnz, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    const int64_t np = np32;
    f->npieces = np;
    int32_t *pfirst = nullptr, *pidx = nullptr, *pidx2 = nullptr, *wcnt = nullptr, *wpfirst = nullptr,
            *wsl = nullptr, *slen = nullptr, *pslot = nullptr, *win_slice = nullptr;
    uint32_t *pkey = nullptr, *pkey2 = nullptr;
    GBK_CUDA(cudaMallocAsync(&pfirst, 4 * (np + 1), s));
    GBK_CUDA(cudaMallocAsync(&pkey, 4 * np, s));
    GBK_CUDA(cudaMallocAsync(&pkey2, 4 * np, s));
    GBK_CUDA(cudaMallocAsync(&pidx, 4 * np, s));
    GBK_CUDA(cudaMallocAsync(&pidx2, 4 * np, s));
    GBK_CUDA(cudaMallocAsync(&pslot, 4 * np, s));
    GBK_CUDA(cudaMallocAsync(&wcnt, 4 * (f->nwin + 1), s));
    GBK_CUDA(cudaMallocAsync(&wpfirst, 4 * (f->nwin + 1), s));
    GBK_CUDA(cudaMallocAsync(&wsl, 4 * (f->nwin + 1), s));
    GBK_CUDA(cudaMallocAsync(&win_slice, 4 * (f->nwin + 1), s));
    GBK_CUDA(cudaMemsetAsync(wcnt, 0, 4 * (f->nwin + 1), s));
    k_sw_pfirst<<<sw_blocks(nnz), 256, 0, s>>>(pflag, pid, nnz, pfirst);
    GBK_LAUNCHED();
    const int32_t nnz32 = (int32_t)nnz;
    GBK_CUDA(cudaMemcpyAsync(pfirst + np, &nnz32, 4, cudaMemcpyHostToDevice, s));
    k_sw_pkey<<<sw_blocks(np), 256, 0, s>>>(pfirst, keys2, np, pkey, pidx);
    GBK_LAUNCHED();
    // pieces by window, then length descending (stable: row order for ties)
    tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, pkey, pkey2, pidx, pidx2, (int)np, 0, 9 + win_bits, s);
    GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(tb, 16), s));
    GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, pkey, pkey2, pidx, pidx2, (int)np, 0, 9 + win_bits, s));
    count_launch(1);
    cudaFreeAsync(tmp, s);
    k_sw_wcount<<<sw_blocks(np), 256, 0, s>>>(pkey2, np, wcnt);
    GBK_LAUNCHED();
    rc = sw_scan_excl(wcnt, wpfirst, f->nwin + 1, s);
    if (rc) return fail(rc);
    k_sw_wslices<<<sw_blocks(f->nwin + 1), 256, 0, s>>>(wcnt, f->nwin, wsl);
    GBK_LAUNCHED();
    rc = sw_scan_excl(wsl, win_slice, f->nwin + 1, s);
    if (rc) return fail(rc);
    int32_t ns32 = 0;
    GBK_CUDA(cudaMemcpyAsync(&ns32, win_slice + f->nwin, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    const int64_t ns = ns32;
    f->nslices = ns;
    GBK_CUDA(cudaMalloc(&f->prow, 4 * 32 * ns));
    GBK_CUDA(cudaMalloc(&f->plen, 2 * 32 * ns));
    GBK_CUDA(cudaMallocAsync(&slen, 4 * (ns + 1), s));
    GBK_CUDA(cudaMemsetAsync(f->prow, 0xff, 4 * 32 * ns, s));
    GBK_CUDA(cudaMemsetAsync(f->plen, 0, 2 * 32 * ns, s));
    k_sw_place<<<sw_blocks(np), 256, 0, s>>>(pkey2, pidx2, np, wpfirst, win_slice, pfirst, keys2, f->prow, f->plen,
                                             slen, pslot);
    GBK_LAUNCHED();
    long long *ent = nullptr, *soff = nullptr;
    GBK_CUDA(cudaMallocAsync(&ent, 8 * (ns + 1), s));
    GBK_CUDA(cudaMallocAsync(&soff, 8 * (ns + 1), s));
    k_sw_steps<<<sw_blocks(ns + 1), 256, 0, s>>>(slen, ns, ent);
    GBK_LAUNCHED();
    size_t eb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, eb, ent, soff, (int)(ns + 1), s);
    GBK_CUDA(cudaMallocAsync(&tmp, std::max<size_t>(eb, 16), s));
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, eb, ent, soff, (int)(ns + 1), s));
    count_launch(1);
    long long padded = 0;
    GBK_CUDA(cudaMemcpyAsync(&padded, soff + ns, 8, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(tmp, s);
    if (padded >= (1ll << 31)) {
        set_error("staged SELL-C: %lld padded entries exceed 2^31", padded);
        return fail(GBK_INSUFFICIENT_SPACE);
    }
    f->padded = padded;
    GBK_CUDA(cudaMalloc(&f->col, 2 * std::max<long long>(padded, 1)));
    GBK_CUDA(cudaMalloc(&f->val, sizeof(T) * std::max<long long>(padded, 1)));
    GBK_CUDA(cudaMemsetAsync(f->col, 0, 2 * std::max<long long>(padded, 1), s));
    GBK_CUDA(cudaMemsetAsync(f->val, 0, sizeof(T) * std::max<long long>(padded, 1), s));
    k_sw_fill<T><<<sw_blocks(nnz), 256, 0, s>>>(keys2, pos2, pflag, pid, pfirst, pslot, soff, a.idx, (const T*)a.val,
                                                nnz, f->col, (T*)f->val);
    GBK_LAUNCHED();
    // work items and shares
    std::vector<int32_t> hslen(ns), hwin(f->nwin + 1), share, hwin_item;
    std::vector<long long> hsoff(ns + 1);
    std::vector<int4> items;
    GBK_CUDA(cudaMemcpyAsync(hslen.data(), slen, 4 * ns, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaMemcpyAsync(hsoff.data(), soff, 8 * (ns + 1), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaMemcpyAsync(hwin.data(), win_slice, 4 * (f->nwin + 1), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    sw_items(hslen, hsoff, hwin, items, hwin_item);
    f->nitems = (int64_t)items.size();
    GBK_CUDA(cudaMalloc(&f->item, sizeof(int4) * std::max<int64_t>(f->nitems, 1)));
    GBK_CUDA(cudaMemcpyAsync(f->item, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, s));
    GBK_CUDA(cudaMemcpyAsync(f->win_item, hwin_item.data(), 4 * hwin_item.size(), cudaMemcpyHostToDevice, s));
    const std::vector<double> cost = sw_model_cost(items, hwin_item);
    sw_cut_shares(cost, num_sms(), share);
    f->nshares = (int32_t)share.size() - 1;
    GBK_CUDA(cudaMalloc(&f->share, 4 * share.size()));
    GBK_CUDA(cudaMemcpyAsync(f->share, share.data(), 4 * share.size(), cudaMemcpyHostToDevice, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    for (void* p : {(void*)keys, (void*)keys2, (void*)pos, (void*)pos2, (void*)vs, (void*)vstart, (void*)pflag,
                    (void*)pid, (void*)pfirst, (void*)pkey, (void*)pkey2, (void*)pidx, (void*)pidx2, (void*)pslot,
                    (void*)wcnt, (void*)wpfirst, (void*)wsl, (void*)slen, (void*)ent, (void*)soff, (void*)win_slice})
        cudaFreeAsync(p, s);  // build temporaries come from the stream-ordered pool
    cudaFree(idx2);
    if (std::is_same<T, float>::value && f->nitems > 0) {
        rc = sw_calibrate(f, cost, share, s);
        if (rc != GBK_SUCCESS) return fail(rc);
        GBK_CUDA(cudaMemsetAsync(f->err, 0, 4, s));
        GBK_CUDA(cudaStreamSynchronize(s));
    }
    *out = f;
    return GBK_SUCCESS;
}

}  // namespace

int build_sellw(const CsrView& a, int dtype, bool reorder, SellW** out, cudaStream_t s) {
    GBK_REQUIRE(a.ncols <= (int64_t)kSwCols * 8388608, GBK_UNSUPPORTED, "staged SELL-C: too many columns");
    return dtype == GBK_F32 ? build_impl<float>(a, reorder, out, s) : build_impl<int32_t>(a, reorder, out, s);
}

int run_sellw(const SellW* f, int sr, int accum, int dtype, const void* x, void* y, cudaStream_t s) {
    if (dtype == GBK_F32) return run_typed<float>(f, sr, accum, (const float*)x, (float*)y, s);
    if (dtype == GBK_I32) return run_typed<int32_t>(f, sr, accum, (const int32_t*)x, (int32_t*)y, s);
    return GBK_UNSUPPORTED;
}

void free_sellw(SellW* f) {
    if (!f) return;
    for (void* p : {(void*)f->col, f->val, (void*)f->item, (void*)f->prow, (void*)f->plen, (void*)f->win_item,
                    (void*)f->share, (void*)f->new_to_old, f->xr, f->tmp, (void*)f->err})
        cudaFree(p);
    delete f;
}

int64_t sellw_padded(const SellW* f) { return f ? f->padded : 0; }

size_t sellw_bytes(const SellW* f) {
    if (!f) return 0;
    return (size_t)f->padded * 6 + (size_t)f->nslices * 32 * 6 + (size_t)f->nitems * 16 +
           (size_t)(f->nwin + f->nshares + 2) * 4 + (f->new_to_old ? (size_t)f->ncols * 8 : 0) +
           (size_t)f->nrows * 4;
}

}  // namespace gbk
