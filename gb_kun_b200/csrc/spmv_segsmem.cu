// CSR_SEG SpMV with the x segment staged in shared memory.
//
// The reference's segmented CSR (src/backend/matrix/seg_csr/build.hpp:23-169,
// src/backend/spmv/spmv_seg.h:8-308) cuts the columns into windows so each
// segment's slice of x stays in cache, computes per-segment row sums and then
// merges them.  Here a window is kSegCols columns, the size of x that fits a
// CTA's shared memory (192 KiB of 4-byte values):
//   * the entries are re-sorted segment-major (then by row, then column), each
//     with a 16-bit column inside its window; the entries of one row inside
//     one segment form a "virtual row";
//   * the entries are cut into 256-entry chunks; lane l of a warp owns entries
//     8 l .. 8 l + 7 of a chunk, and a 16-bit group record per 8 entries holds
//     their virtual-row start bits and the number of starts earlier in the
//     chunk, so a lane knows its virtual rows without a scan;
//   * 148 persistent CTAs (one per SM, 1024 threads) take shares of whole
//     chunks of equal cost: first a model (entries, virtual rows and windows
//     weighted by measured costs), then calibrated at build time from each
//     CTA's timed share; for each segment it touches a CTA copies that window
//     of x into shared memory once (asynchronous copies into bank-swizzled
//     positions; the stored columns are already the swizzled positions);
//   * its warps walk whole chunks: 16-byte column / value loads one chunk
//     ahead, eight gathers from shared memory per lane, each lane's tail sum,
//     ONE segmented warp scan per 256 entries for the runs that cross lanes,
//     then a forward pass that writes every closed run's sum to a per-warp
//     buffer in run order;
//   * the warp folds those sums into y, 32 runs at a time, with one atomic of
//     the semiring's add each (float / int add, int / float minimum, or a
//     store of 1 for the logical-or semirings), so there is no merge pass.
// Float sums therefore add in an order that varies between runs (within the
// FP32 tolerance); integer and min / or results are exact.  Semirings whose
// add is not associative fall back to the CSR kernels.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace gbk {

constexpr int kSegCols = 49152;  // x values per staged window (192 KiB of 4-byte values)
constexpr int kSegThreads = 1024;
constexpr int kLaneEntries = 8;                  // entries per lane of a chunk
constexpr int kChunk = 32 * kLaneEntries;        // entries per warp chunk
constexpr int kGroups = kChunk / kLaneEntries;   // group records per chunk (one per lane)
// run sums of one chunk: up to kChunk closed runs and the one left open,
// padded to 16 bytes
constexpr int kRunSlots = kChunk + 8;
// dynamic shared memory of the SpMV kernel: the x window and one run-sum
// buffer per warp (4-byte values)
constexpr size_t kSegSmemBytes = 4 * ((size_t)kSegCols + (size_t)(kSegThreads / 32) * kRunSlots);

// Window position of column c (c < 65536) in shared memory: the column's
// bank bits XOR the three higher 5-bit groups, a permutation inside each
// 32-column block.  Power-law graphs put most entries on columns whose low
// bits are zero; without the swizzle those all fall in bank 0.
__host__ __device__ __forceinline__ uint32_t window_pos(uint32_t c) {
    return c ^ (((c >> 5) ^ (c >> 10) ^ (c >> 15)) & 31u);
}

struct SegSmem {
    int64_t nrows = 0, ncols = 0, nnz = 0, nvrows = 0;
    int64_t nchunks = 0;
    int32_t nseg = 0;
    uint16_t* col = nullptr;       // window position of the column (window_pos), nchunks * kChunk (zero padded)
    void* val = nullptr;           // nchunks * kChunk (zero padded)
    uint16_t* grp = nullptr;       // per 8 entries: (virtual-row starts earlier in the chunk) << 8 | start bits
    int32_t* cvr = nullptr;        // nchunks + 1: virtual row open just before entry kChunk * q (-1 at 0)
    int32_t* vrow = nullptr;       // original row of each virtual row
    int32_t* seg_start = nullptr;  // nseg + 1 entry offsets
    int32_t nshares = 0;           // CTAs of the SpMV launch (one per SM)
    int32_t* share = nullptr;      // nshares + 1 entry offsets of the CTAs' shares (chunk aligned)
    void* tmp = nullptr;           // nrows: the product before the accumulator
    int32_t* err = nullptr;        // first failed index check seen by the kernel (0 = none)
    bool check = true;             // read err back after the first launch
};

namespace {

// key = (window << 32) | row, value = entry position; one thread per entry,
// its row by binary search in the row pointers (balanced over hub rows)
__global__ void k_ss_keys(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx, int64_t n, int64_t nnz,
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
    keys[e] = ((unsigned long long)(idx[e] / kSegCols) << 32) | (unsigned long long)lo;
    pos[e] = (int32_t)e;
}

template <typename T>
__global__ void k_ss_fill(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ pos,
                          const int32_t* __restrict__ idx, const T* __restrict__ v, int64_t nnz,
                          uint16_t* __restrict__ col, T* __restrict__ val, int32_t* __restrict__ flag,
                          int32_t* __restrict__ seg_start) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    const unsigned long long k = keys[i];
    const int32_t seg = (int32_t)(k >> 32);
    const int32_t e = pos[i];
    col[i] = (uint16_t)window_pos((uint32_t)(idx[e] - seg * kSegCols));
    val[i] = v[e];
    flag[i] = (i == 0) || (keys[i - 1] != k);
    if (i == 0 || (int32_t)(keys[i - 1] >> 32) != seg) seg_start[seg] = (int32_t)i;
}

__global__ void k_ss_vrows(const unsigned long long* __restrict__ keys, const int32_t* __restrict__ flag,
                           const int32_t* __restrict__ vid, int64_t nnz, int32_t* __restrict__ vrow) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    if (flag[i]) vrow[vid[i]] = (int32_t)(keys[i] & 0xffffffffu);
}

// Group records and chunk starts from the start flags and their exclusive
// scan vid (vid[i] = virtual rows starting before entry i, vid[nnz] = total).
__global__ void k_ss_groups(const int32_t* __restrict__ flag, const int32_t* __restrict__ vid, int64_t nnz,
                            int64_t ngroups, uint16_t* __restrict__ grp) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    const int64_t e0 = g * kLaneEntries, cb = (g / kGroups) * kChunk;
    unsigned bits = 0;
    for (int i = 0; i < kLaneEntries; ++i)
        if (e0 + i < nnz && flag[e0 + i]) bits |= 1u << i;
    const int32_t before = vid[min(e0, nnz)] - vid[min(cb, nnz)];  // < kChunk
    grp[g] = (uint16_t)(((unsigned)before << 8) | bits);
}

__global__ void k_ss_cvr(const int32_t* __restrict__ vid, int64_t nnz, int64_t nchunks, int32_t* __restrict__ cvr) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q > nchunks) return;
    cvr[q] = vid[min(q * kChunk, nnz)] - 1;
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

// Does folding v into y change anything?  (The identity of the add never
// does, so empty and masked-out runs cost no atomic.)
template <int SR, typename T>
__device__ __forceinline__ bool changes(T v) {
    using S = Semiring<SR, T>;
    constexpr int cls = AddClass<SR>::value;
    if constexpr (cls == 1)
        return v < S::identity();
    else
        return v != T(0);
}

// atomic fold of one virtual row's sum into out[r] by the semiring's add
template <int SR, typename T>
__device__ __forceinline__ void fold_into(T* out, int32_t r, T v) {
    constexpr int cls = AddClass<SR>::value;
    if constexpr (cls == 0)
        atomic_add_any(out + r, v);
    else if constexpr (cls == 1)
        atomic_min_any(out + r, v);
    else
        out[r] = T(1);
}

// Index checks: a virtual row, row or window column out of range is recorded
// in *err (first one wins) and the access skipped or clamped, so a malformed
// structure reports an error instead of touching memory it does not own.
__device__ __forceinline__ void ss_flag(int32_t* err, int32_t code) { atomicCAS(err, 0, code); }

template <int SR, typename T>
__device__ __forceinline__ void ss_emit(T* out, int32_t r, T v, int64_t nrows, int32_t* err) {
    if (!changes<SR, T>(v)) return;
    if (r < 0 || r >= nrows)
        ss_flag(err, 2);
    else
        fold_into<SR, T>(out, r, v);
}

template <typename T> __device__ __forceinline__ T from_bits(uint32_t u);
template <> __device__ __forceinline__ float from_bits<float>(uint32_t u) { return __uint_as_float(u); }
template <> __device__ __forceinline__ int32_t from_bits<int32_t>(uint32_t u) { return (int32_t)u; }

// One warp's share of the chunks [qa, qb) of the staged segment, restricted
// to the entries [a, b) (the first and last chunk may hold entries of a
// neighbouring segment or of another CTA's share: those add the identity, but
// their virtual-row starts still count, so the row numbering stays global).
// The warps of the CTA take chunks one at a time from a shared counter, so a
// warp with costly chunks does not hold the others at the next window.
//
// Every chunk stands alone: the lanes' products; each lane's tail (the sum
// after its last start); a segmented warp scan of the tails gives the run
// coming into every lane; a forward pass from that value gives the sum of
// every run a start closes, which the lane writes to the warp's buffer at the
// run's index in the chunk (run k of the chunk is virtual row cvr + k; the
// run still open at the chunk's end is run nrun).  The warp then folds runs
// lane, lane + 32, ... into y, their rows loaded at the start of the chunk.
// Failed index checks are collected per lane and reported once at the end.
template <int SR, typename T>
__device__ __forceinline__ void ss_warp_chunks(const uint4* __restrict__ col8, const uint4* __restrict__ val4,
                                               const uint16_t* __restrict__ grp, const int32_t* __restrict__ cvr,
                                               const int32_t* __restrict__ vrow, const T* xs, T* buf, int w,
                                               int64_t qa, int64_t qb, int64_t a, int64_t b, int* next, T* out,
                                               int64_t nvrows, int64_t nrows, int32_t* err) {
    using S = Semiring<SR, T>;
    constexpr int kRowsAhead = 2;  // runs per lane whose rows are loaded at the start of a chunk
    const unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned le = (lane == 31) ? kAll : ((2u << lane) - 1u);
    const unsigned wl = (unsigned)(((w + 31) & ~31) - 1);  // last staged position of the window
    const unsigned wl2 = wl | (wl << 16);
    const uint32_t nvr = (uint32_t)nvrows, nr = (uint32_t)nrows;  // both < 2^31
    bool bad_col = false, bad_row = false;
    // chunk and entry numbers fit 32 bits (nnz < 2^31)
    const int32_t qa32 = (int32_t)qa, qb32 = (int32_t)qb, a32 = (int32_t)a, b32 = (int32_t)b;
    auto grab = [&]() -> int32_t {
        int t = 0;
        if (lane == 0) t = atomicAdd(next, 1);
        return qa32 + __shfl_sync(kAll, t, 0);
    };
    int32_t q = grab();
    if (q >= qb32) return;
    uint4 cn = __ldcs(col8 + q * kGroups + lane);
    uint4 an = __ldcs(val4 + q * 2 * kGroups + 2 * lane), bn = __ldcs(val4 + q * 2 * kGroups + 2 * lane + 1);
    uint32_t gn = __ldcs(grp + q * kGroups + lane);
    int32_t vn = __ldg(cvr + q);
    for (;;) {
        const int32_t qn = grab();
        const uint4 c = cn, va = an, vb = bn;
        const uint32_t g = gn;
        const int32_t cv = vn;
        if (qn < qb32) {  // the next chunk's loads go out before this chunk's work
            cn = __ldcs(col8 + qn * kGroups + lane);
            an = __ldcs(val4 + qn * 2 * kGroups + 2 * lane);
            bn = __ldcs(val4 + qn * 2 * kGroups + 2 * lane + 1);
            gn = __ldcs(grp + qn * kGroups + lane);
            vn = __ldg(cvr + qn);
        }
        const uint32_t hb = g & 0xffu;      // entries of this lane that start a virtual row
        const uint32_t before = g >> 8;     // starts in the chunk before this lane's entries
        const int nrun = (int)__shfl_sync(kAll, before + __popc(hb), 31);  // runs the chunk's starts close
        // rows of the first runs this lane folds (runs 0 .. nrun)
        int32_t rr[kRowsAhead];
#pragma unroll
        for (int k = 0; k < kRowsAhead; ++k) {
            const uint32_t vr = (uint32_t)(cv + lane + 32 * k);
            rr[k] = (lane + 32 * k <= nrun && vr < nvr) ? __ldg(vrow + vr) : -1;
        }
        // a ragged chunk: entries outside [a, b) (another window's columns, or
        // another share) read position 0 and add the identity
        const int32_t cb = q * kChunk, e0 = cb + lane * kLaneEntries;
        const bool ragged = cb < a32 || cb + kChunk > b32;
        uint32_t cr[4] = {c.x, c.y, c.z, c.w};
        if (ragged) {
#pragma unroll
            for (int i = 0; i < kLaneEntries; ++i)
                if (e0 + i < a32 || e0 + i >= b32) cr[i >> 1] &= (i & 1) ? 0x0000ffffu : 0xffff0000u;
        }
        // products; positions are clamped into the window and one outside it
        // is reported
        const uint32_t cmax = __vmaxu2(__vmaxu2(cr[0], cr[1]), __vmaxu2(cr[2], cr[3]));
        bad_col |= (cmax & 0xffffu) > wl || (cmax >> 16) > wl;
        const uint32_t vw[kLaneEntries] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
        T p[kLaneEntries];
#pragma unroll
        for (int i = 0; i < kLaneEntries; ++i) {
            const uint32_t cw = __vminu2(cr[i >> 1], wl2);
            const uint32_t ci = (i & 1) ? (cw >> 16) : (cw & 0xffffu);
            p[i] = S::mul(from_bits<T>(vw[i]), xs[ci]);
        }
        if (ragged) {
#pragma unroll
            for (int i = 0; i < kLaneEntries; ++i)
                if (e0 + i < a32 || e0 + i >= b32) p[i] = S::identity();
        }
        // this lane's tail: the entries from its last start on (all of them
        // when it has none)
        const int last = hb ? 31 - __clz(hb) : 0;
        T tail = S::identity();
#pragma unroll
        for (int i = 0; i < kLaneEntries; ++i)
            if (i >= last) tail = S::add(tail, p[i]);
        // segmented warp scan of the tails: s = the run open after this lane,
        // including earlier lanes when no start lies between
        const unsigned hle = __ballot_sync(kAll, hb != 0) & le;
        const int first = hle ? 31 - __clz(hle) : 0;  // last lane at or before this one with a start
        T s = tail;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T o = __shfl_up_sync(kAll, s, d);
            if (lane - d >= first) s = S::add(s, o);
        }
        T acc = __shfl_up_sync(kAll, s, 1);  // the run open before this lane
        if (lane == 0) acc = S::identity();
        // forward pass: a start at i closes the run summed so far; its sum
        // goes to the buffer at the run's index in the chunk
        T* slot = buf + before;
#pragma unroll
        for (int i = 0; i < kLaneEntries; ++i) {
            if ((hb >> i) & 1u) {
                *slot++ = acc;
                acc = p[i];
            } else {
                acc = S::add(acc, p[i]);
            }
        }
        if (lane == 31) *slot = acc;  // the run open at the chunk's end (slot = buf + nrun)
        __syncwarp();
        // fold the runs
#pragma unroll
        for (int k = 0; k < kRowsAhead; ++k) {  // (slots past nrun hold stale sums and fold nothing)
            const int j = lane + 32 * k;
            const T v = buf[j];
            const bool fold = j <= nrun && changes<SR, T>(v);
            const bool ok = (uint32_t)rr[k] < nr;
            if (fold && ok) fold_into<SR, T>(out, rr[k], v);
            bad_row |= fold && !ok;
        }
        for (int j = lane + 32 * kRowsAhead; j <= nrun; j += 32) {  // chunks with 64 runs or more
            const T v = buf[j];
            if (changes<SR, T>(v)) {
                const uint32_t vr = (uint32_t)(cv + j);
                const int32_t r = vr < nvr ? __ldg(vrow + vr) : -1;
                if ((uint32_t)r < nr)
                    fold_into<SR, T>(out, r, v);
                else
                    bad_row = true;
            }
        }
        __syncwarp();  // the buffer is read before the next chunk writes it
        if (qn >= qb32) break;
        q = qn;
    }
    if (bad_col) ss_flag(err, 1);
    if (bad_row) ss_flag(err, 2);
}

// Copy w values of x into their swizzled shared-memory positions with 4-byte
// asynchronous copies (all of a thread's copies in flight, no registers
// held).  Returns once this thread's copies have landed; the caller's
// barrier publishes them.
template <typename T>
__device__ __forceinline__ void stage_window(T* xs, const T* src, int w) {
    static_assert(sizeof(T) == 4, "4-byte values");
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(xs);
    for (int i = threadIdx.x; i < w; i += blockDim.x)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst + 4u * window_pos((uint32_t)i)),
                     "l"(src + i)
                     : "memory");
    asm volatile("cp.async.wait_all;" ::: "memory");
}

template <int SR, typename T>
__global__ void __launch_bounds__(kSegThreads, 1)
    k_segsmem(const uint16_t* __restrict__ col, const T* __restrict__ val, const uint16_t* __restrict__ grp,
              const int32_t* __restrict__ cvr, const int32_t* __restrict__ vrow,
              const int32_t* __restrict__ seg_start, const int32_t* __restrict__ share, int32_t nseg,
              int64_t ncols, int64_t nvrows, int64_t nrows, const T* __restrict__ x, T* out, int32_t* err,
              long long* clk) {
    extern __shared__ __align__(16) unsigned char ss_smem[];
    T* xs = reinterpret_cast<T*>(ss_smem);
    const int warp = threadIdx.x >> 5;
    T* buf = xs + kSegCols + warp * kRunSlots;  // this warp's run sums
    __shared__ int next_chunk;                  // chunks of the segment part handed out so far
    const long long t0 = clock64();
    const int64_t c0 = share[blockIdx.x], c1 = share[blockIdx.x + 1];
    if (c0 >= c1) {  // the whole block leaves together
        if (clk && threadIdx.x == 0) clk[blockIdx.x] = 0;
        return;
    }
    int lo = 0, hi = nseg;  // last segment starting at or before c0
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (seg_start[mid] <= c0)
            lo = mid;
        else
            hi = mid;
    }
    const uint4* col8 = reinterpret_cast<const uint4*>(col);
    const uint4* val4 = reinterpret_cast<const uint4*>(val);
    for (int s = lo; s < nseg && seg_start[s] < c1; ++s) {
        const int64_t a = max(c0, (int64_t)seg_start[s]), b = min(c1, (int64_t)seg_start[s + 1]);
        if (a >= b) continue;
        __syncthreads();  // the previous window's readers are done
        if (threadIdx.x == 0) next_chunk = 0;
        const int64_t col0 = (int64_t)s * kSegCols;
        const int w = (int)min((int64_t)kSegCols, ncols - col0);
        stage_window(xs, x + col0, w);
        __syncthreads();
        // y's initialisation (the kernel before this one on the stream) has
        // finished before the first fold.  Launched with programmatic stream
        // serialisation, everything above overlaps it; otherwise a no-op.
        asm volatile("griddepcontrol.wait;" ::: "memory");
        const int64_t qa = a / kChunk, qb = (b + kChunk - 1) / kChunk;
        ss_warp_chunks<SR, T>(col8, val4, grp, cvr, vrow, xs, buf, w, qa, qb, a, b, &next_chunk, out, nvrows, nrows,
                              err);
    }
    if (clk) {  // calibration launches: the block's time in SM cycles
        __syncthreads();
        if (threadIdx.x == 0) clk[blockIdx.x] = clock64() - t0;
    }
}

template <int SR, typename T>
// overlap_prev: the kernel before this launch on the stream is y's
// initialisation, which calls griddepcontrol.launch_dependents; this launch
// may then start (and stage its first window) while it runs.
int launch_segsmem(const SegSmem* f, const T* x, T* out, long long* clk, bool overlap_prev, cudaStream_t s) {
    static bool attr = false;  // one per instantiation
    if (!attr) {
        GBK_CUDA(cudaFuncSetAttribute(k_segsmem<SR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSegSmemBytes));
        attr = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)f->nshares);
    cfg.blockDim = dim3(kSegThreads);
    cfg.dynamicSmemBytes = kSegSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    la[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = la;
    cfg.numAttrs = overlap_prev ? 1 : 0;
    GBK_CUDA(cudaLaunchKernelEx(&cfg, k_segsmem<SR, T>, (const uint16_t*)f->col, (const T*)f->val,
                                (const uint16_t*)f->grp, (const int32_t*)f->cvr, (const int32_t*)f->vrow,
                                (const int32_t*)f->seg_start, (const int32_t*)f->share, f->nseg, f->ncols, f->nvrows,
                                f->nrows, x, out, f->err, clk));
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

template <typename T>
__global__ void k_ss_init(T* out, int64_t n, T v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v;
}

// y = the add's identity before the folds: grid-stride 16-byte stores (the
// caller's y may be only 4-byte aligned: the head and tail go one by one)
template <typename T>
__global__ void k_ss_identity(T* __restrict__ out, int64_t n, T v) {
    asm volatile("griddepcontrol.launch_dependents;");  // the SpMV kernel may start its prologue
    const int64_t lead = (int64_t)((16 - (reinterpret_cast<uintptr_t>(out) & 15)) & 15) / 4;
    const int64_t head = lead < n ? lead : n;
    const int64_t n4 = (n - head) / 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint4 w;
    w.x = w.y = w.z = w.w = *reinterpret_cast<const uint32_t*>(&v);
    uint4* o4 = reinterpret_cast<uint4*>(out + head);
    for (int64_t i = t; i < n4; i += stride) o4[i] = w;
    if (t < head) out[t] = v;
    const int64_t tail = head + 4 * n4 + t;
    if (tail < n) out[tail] = v;
}

template <typename T>
__global__ void k_ss_accum(T* __restrict__ y, const T* __restrict__ t, int64_t n, int accum) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = binop<T>(accum, y[i], t[i]);
}

unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

// Relative costs of the work a CTA does, in entries: a virtual row costs an
// atomic fold and a row lookup, a window a 192 KiB copy and two barriers.
// Swept on R-MAT scale 22 (0 - 5 per virtual row, 0 - 65536 per window; equal
// entry shares ran 1.55x slower than these); Erdos-Renyi, whose cost is
// uniform, is indifferent.  GBK_SEG_VROW_COST / GBK_SEG_WINDOW_COST override.
constexpr double kVrowCost = 2.0;
constexpr double kWindowCost = 16384.0;

double env_weight(const char* name, double dflt) {
    const char* e = std::getenv(name);
    return e ? std::atof(e) : dflt;
}

// Modelled cost of the entries before chunk q (q = 0 .. nchunks): entries +
// virtual rows + windows begun, in entries.
std::vector<double> model_cost(const std::vector<int32_t>& cvr, const std::vector<int32_t>& seg_start, int64_t nnz) {
    const double wv = env_weight("GBK_SEG_VROW_COST", kVrowCost), ww = env_weight("GBK_SEG_WINDOW_COST", kWindowCost);
    const int64_t nch = (int64_t)cvr.size() - 1;
    std::vector<double> cost(nch + 1);
    size_t sg = 0;
    int64_t begun = 0;  // non-empty segments starting at or before entry e
    for (int64_t q = 0; q <= nch; ++q) {
        const int64_t e = std::min<int64_t>(q * kChunk, nnz);
        for (; sg + 1 < seg_start.size() && seg_start[sg] <= e; ++sg)
            if (seg_start[sg] < seg_start[sg + 1]) ++begun;
        cost[q] = (double)e + wv * (double)(cvr[q] + 1) + ww * (double)begun;
    }
    return cost;
}

// Cut the chunks into nsh shares of equal weight (w: non-decreasing weight of
// the chunks before q): share b is entries [share[b], share[b + 1]), chunk
// aligned except the end (nnz).
void cut_shares(const std::vector<double>& w, int64_t nnz, int nsh, std::vector<int32_t>& share) {
    const int64_t nch = (int64_t)w.size() - 1;
    share.assign(nsh + 1, 0);
    int64_t q = 0;
    for (int b = 1; b < nsh; ++b) {
        const double target = w[nch] * b / nsh;
        while (q < nch && w[q] < target) ++q;
        share[b] = (int32_t)std::min<int64_t>(q * kChunk, nnz);
    }
    share[nsh] = (int32_t)nnz;
}

// Calibrated shares: time every CTA's share (plus-times over x = 1, SM
// cycles, the median of three warm launches), spread each share's time over
// its chunks by the modelled cost, average with the previous rounds'
// estimate and cut again at equal time; the shares whose slowest CTA was
// fastest over all rounds are kept.  The model alone leaves the slowest CTA
// 1.2 - 1.5x above the mean on power-law graphs, and a single round's cut
// moves with timing noise.
constexpr int kCalibrationRounds = 8;
constexpr int kCalibrationReps = 3;

int calibrate_shares(SegSmem* f, const std::vector<double>& cost, std::vector<int32_t>& share, cudaStream_t s) {
    const int nsh = f->nshares;
    const int64_t nch = (int64_t)cost.size() - 1;
    float* x1 = nullptr;
    long long* clk = nullptr;
    GBK_CUDA(cudaMalloc(&x1, sizeof(float) * std::max<int64_t>(f->ncols, 1)));
    GBK_CUDA(cudaMalloc(&clk, sizeof(long long) * nsh));
    k_ss_init<float><<<blocks(f->ncols), 256, 0, s>>>(x1, f->ncols, 1.0f);
    GBK_LAUNCHED();
    std::vector<long long> t(nsh);
    std::vector<std::vector<long long>> reps(kCalibrationReps, std::vector<long long>(nsh));
    std::vector<double> w(nch + 1), wavg;
    std::vector<int32_t> best = share;
    long long best_max = -1;
    int rc = GBK_SUCCESS;
    for (int round = 0; round < kCalibrationRounds && rc == GBK_SUCCESS; ++round) {
        rc = launch_segsmem<GBK_PLUS_TIMES, float>(f, x1, (float*)f->tmp, clk, false, s);  // warm-up
        for (int rep = 0; rep < kCalibrationReps && rc == GBK_SUCCESS; ++rep) {
            rc = launch_segsmem<GBK_PLUS_TIMES, float>(f, x1, (float*)f->tmp, clk, false, s);
            if (rc != GBK_SUCCESS) break;
            GBK_CUDA(cudaMemcpyAsync(reps[rep].data(), clk, sizeof(long long) * nsh, cudaMemcpyDeviceToHost, s));
        }
        if (rc != GBK_SUCCESS) break;
        GBK_CUDA(cudaStreamSynchronize(s));
        long long tmax = 0;
        for (int b = 0; b < nsh; ++b) {
            long long v[kCalibrationReps];
            for (int r = 0; r < kCalibrationReps; ++r) v[r] = reps[r][b];
            std::sort(v, v + kCalibrationReps);
            t[b] = v[kCalibrationReps / 2];
            tmax = std::max(tmax, t[b]);
        }
        if (best_max < 0 || tmax < best_max) {
            best_max = tmax;
            best = share;
        }
        double tsum = 0, csum = 0;
        for (int b = 0; b < nsh; ++b) {
            const int64_t q0 = (share[b] + kChunk - 1) / kChunk, q1 = (share[b + 1] + kChunk - 1) / kChunk;
            if (q1 > q0 && t[b] > 0) {
                tsum += (double)t[b];
                csum += cost[q1] - cost[q0];
            }
        }
        if (tsum <= 0 || csum <= 0) break;
        double acc = 0;
        w[0] = 0;
        for (int b = 0; b < nsh; ++b) {
            const int64_t q0 = (share[b] + kChunk - 1) / kChunk, q1 = (share[b + 1] + kChunk - 1) / kChunk;
            if (q1 <= q0) continue;
            const double cb = cost[q1] - cost[q0];
            const double tb = t[b] > 0 ? (double)t[b] : cb * tsum / csum;
            for (int64_t q = q0 + 1; q <= q1; ++q) w[q] = acc + tb * (cost[q] - cost[q0]) / cb;
            acc += tb;
        }
        if (wavg.empty()) {
            wavg = w;
        } else {
            for (int64_t q = 0; q <= nch; ++q) wavg[q] = 0.5 * (wavg[q] + w[q]);
        }
        cut_shares(wavg, f->nnz, nsh, share);
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
int build_impl(const CsrView& a, SegSmem** out, cudaStream_t s) {
    SegSmem* f = new SegSmem();
    f->nrows = a.nrows;
    f->ncols = a.ncols;
    f->nnz = a.nnz;
    f->nseg = (int32_t)std::max<int64_t>(1, (a.ncols + kSegCols - 1) / kSegCols);
    const int64_t nnz = a.nnz;
    f->nchunks = std::max<int64_t>(1, (nnz + kChunk - 1) / kChunk);
    const int64_t padded = f->nchunks * kChunk, ngroups = f->nchunks * kGroups;
    auto fail = [&](int rc) {
        free_segsmem(f);
        return rc;
    };
    if (cudaMalloc(&f->col, 2 * padded) || cudaMalloc(&f->val, sizeof(T) * padded) ||
        cudaMalloc(&f->grp, 2 * ngroups) || cudaMalloc(&f->cvr, 4 * (f->nchunks + 1)) ||
        cudaMalloc(&f->seg_start, 4 * (f->nseg + 1)) ||
        cudaMalloc(&f->tmp, sizeof(T) * std::max<int64_t>(a.nrows, 1)) || cudaMalloc(&f->err, 4))
        return fail(cuda_fail(cudaGetLastError(), "segmented format allocation", __FILE__, __LINE__));
    if (cudaMemsetAsync(f->col, 0, 2 * padded, s) || cudaMemsetAsync(f->val, 0, sizeof(T) * padded, s) ||
        cudaMemsetAsync(f->grp, 0, 2 * ngroups, s) || cudaMemsetAsync(f->cvr, 0xff, 4 * (f->nchunks + 1), s) ||
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
        k_ss_keys<<<blocks(a.nnz), 256, 0, s>>>(a.ptr, a.idx, a.nrows, a.nnz, keys, pos);
        GBK_LAUNCHED();
        int seg_bits = 1;
        while ((1ll << seg_bits) < f->nseg) ++seg_bits;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, pos, pos2, (int)nnz, 32, 32 + seg_bits, s);
        void* tmp = nullptr;
        GBK_CUDA(cudaMalloc(&tmp, std::max<size_t>(tb, 16)));
        GBK_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, pos, pos2, (int)nnz, 32, 32 + seg_bits, s));
        count_launch(1);
        GBK_CUDA(cudaMemsetAsync(f->seg_start, 0xff, 4 * (f->nseg + 1), s));
        GBK_CUDA(cudaMemsetAsync(flag + nnz, 0, 4, s));
        k_ss_fill<T><<<blocks(nnz), 256, 0, s>>>(keys2, pos2, a.idx, (const T*)a.val, nnz, f->col, (T*)f->val, flag,
                                                 f->seg_start);
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
        k_ss_vrows<<<blocks(nnz), 256, 0, s>>>(keys2, flag, vid, nnz, f->vrow);
        GBK_LAUNCHED();
        k_ss_groups<<<blocks(ngroups), 256, 0, s>>>(flag, vid, nnz, ngroups, f->grp);
        GBK_LAUNCHED();
        k_ss_cvr<<<blocks(f->nchunks + 1), 256, 0, s>>>(vid, nnz, f->nchunks, f->cvr);
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
    // the CTAs' shares
    std::vector<int32_t> cvr(f->nchunks + 1), share;
    GBK_CUDA(cudaMemcpyAsync(cvr.data(), f->cvr, 4 * (f->nchunks + 1), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    const std::vector<double> cost = model_cost(cvr, ss, nnz);
    cut_shares(cost, nnz, num_sms(), share);
    f->nshares = (int32_t)share.size() - 1;
    GBK_CUDA(cudaMalloc(&f->share, 4 * share.size()));
    GBK_CUDA(cudaMemcpyAsync(f->share, share.data(), 4 * share.size(), cudaMemcpyHostToDevice, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    if (std::is_same<T, float>::value && nnz > 0) {
        const int rc = calibrate_shares(f, cost, share, s);
        if (rc != GBK_SUCCESS) return fail(rc);
        GBK_CUDA(cudaMemsetAsync(f->err, 0, 4, s));
    }
    *out = f;
    return GBK_SUCCESS;
}

template <int SR, typename T>
int run_impl(const SegSmem* f, int accum, const T* x, T* y, cudaStream_t s) {
    using S = Semiring<SR, T>;
    T* out = accum == GBK_OP_SECOND ? y : (T*)f->tmp;
    if (f->nrows > 0) {
        const unsigned nb = (unsigned)std::min<int64_t>((f->nrows / 4 + 255) / 256 + 1, 8 * num_sms());
        k_ss_identity<T><<<nb, 256, 0, s>>>(out, f->nrows, S::identity());
        GBK_LAUNCHED();
    }
    if (f->nnz > 0) {
        const int rc = launch_segsmem<SR, T>(f, x, out, nullptr, f->nrows > 0, s);
        if (rc != GBK_SUCCESS) return rc;
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
    cudaFree(f->grp);
    cudaFree(f->cvr);
    cudaFree(f->vrow);
    cudaFree(f->seg_start);
    cudaFree(f->share);
    cudaFree(f->tmp);
    cudaFree(f->err);
    delete f;
}

size_t segsmem_bytes(const SegSmem* f) {
    if (!f) return 0;
    return (size_t)f->nchunks * kChunk * 6 + (size_t)f->nchunks * kGroups * 2 + (size_t)(f->nchunks + 1) * 4 +
           (size_t)f->nvrows * 4 + (size_t)(f->nseg + 1) * 4 + (size_t)(f->nshares + 1) * 4 + (size_t)f->nrows * 4;
}

}  // namespace gbk
