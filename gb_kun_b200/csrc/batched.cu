// Batched BFS / PPR / SSSP engines and their one-shot C entry points.
//
// Semantics follow the single-source algorithms of the reference, one lane
// per source: BFS levels as bfs_blast (algorithms/bfs/bfs.hpp:93-142; source
// = 1, unreached = 0, edges followed along CSR rows); PPR as the reference's
// page_rank_sinks iteration (algorithms/pr/pr.hpp:20-153) with the teleport
// and the sink mass sent to the seed; SSSP distances as
// sssp_bellman_ford_blast (algorithms/sssp/sssp_blast.hpp:8-72) with integer
// weights.  The batching, the bit packing and the graph-driven loop have no
// counterpart in the reference.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>

#include "batched.h"
#include "common.cuh"

namespace gbk {
namespace {

constexpr int kBT = 256;  // threads per block of the persistent kernels
constexpr int kBfsPiece = 256;  // entries per piece of a long row in the batched BFS push
constexpr unsigned kFull = 0xffffffffu;

int persistent_blocks(const void* kern, int threads) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * num_sms();
}

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long x) {
    const unsigned lo = __reduce_or_sync(kFull, (unsigned)x);
    const unsigned hi = __reduce_or_sync(kFull, (unsigned)(x >> 32));
    return ((unsigned long long)hi << 32) | lo;
}
__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    return x;
}

using LoopBody = std::function<int(cudaStream_t, cudaGraphConditionalHandle)>;

// A graph whose only root node is a `while` conditional; its body is one
// iteration, captured from a stream.  With GBK_BATCH_HOST_LOOP=1 in the
// environment (for profilers that do not follow conditional graph nodes) the
// same body kernels are launched from a host loop instead, one iteration per
// round trip, stopping by the rules the control kernels apply.
struct LoopGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle = 0;
    LoopBody body;
    bool host = false;
    ~LoopGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

int build_loop(LoopGraph& g, LoopBody body) {
    g.body = std::move(body);
    const char* env = getenv("GBK_BATCH_HOST_LOOP");
    g.host = env && env[0] == '1';
    if (g.host) return GBK_SUCCESS;
    GBK_CUDA(cudaGraphCreate(&g.graph, 0));
    GBK_CUDA(cudaGraphConditionalHandleCreate(&g.handle, g.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = g.handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    GBK_CUDA(cudaGraphAddNode(&node, g.graph, nullptr, 0, &p));
    cudaGraph_t bodyg = p.conditional.phGraph_out[0];
    cudaStream_t cs;
    GBK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return cuda_fail(e, "cudaStreamBeginCaptureToGraph", __FILE__, __LINE__);
    }
    const int rc = g.body(cs, g.handle);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    GBK_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    return GBK_SUCCESS;
}

// One launch of the loop; the status lands in h_status on stream s.
int run_loop(LoopGraph& g, BatchStatus* d_status, BatchStatus* h_status, int budget, bool stop_on_finish,
             cudaStream_t s) {
    if (!g.host) {
        GBK_CUDA(cudaGraphLaunch(g.exec, s));
        GBK_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
        return GBK_SUCCESS;
    }
    GBK_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    const unsigned long long fin0 = h_status->finished;
    for (int i = 0; i < budget && h_status->active; ++i) {
        const int rc = g.body(s, 0);
        if (rc) return rc;
        GBK_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        if (stop_on_finish && (h_status->finished & ~fin0)) break;
    }
    return GBK_SUCCESS;
}

// ----------------------------------------------------------------------------
// work items for the column-lane kernels: each CSR row is cut into pieces of
// at most `C` entries; rows of more than one piece ("split" rows) write their
// piece sums to slots that a fixup pass adds in piece order.

struct RowItems {
    int64_t nitems = 0, nsplit = 0, nslots = 0;
    int32_t* item_row = nullptr;     // first row
    int32_t* item_end = nullptr;     // one past the last row
    int32_t* item_beg = nullptr;     // first edge
    int32_t* item_ee = nullptr;      // one past the last edge
    int32_t* item_slot = nullptr;    // >= 0: piece of a split row, its partial-sum slot
    int32_t* split_row = nullptr;    // nsplit
    int32_t* split_first = nullptr;  // nsplit + 1 slot offsets
    void release() {
        cudaFree(item_row);
        cudaFree(item_end);
        cudaFree(item_beg);
        cudaFree(item_ee);
        cudaFree(item_slot);
        cudaFree(split_row);
        cudaFree(split_first);
        *this = RowItems{};
    }
};

// Rows of more than C entries are cut into pieces of C.  Without grouping
// every other row is one item; with grouping, consecutive short rows share
// an item until the edge offset crosses a multiple of C or 32 rows are taken
// (so an item holds at most 2C edges and 32 rows).
__device__ __forceinline__ bool group_start(const int32_t* __restrict__ rp, int64_t v, int C) {
    if (v == 0 || (v & 31) == 0) return true;
    const int32_t prev = rp[v] - rp[v - 1];
    return prev > C || rp[v] / C != rp[v - 1] / C;
}

__global__ void k_item_counts(const int32_t* __restrict__ rp, int64_t n, int C, int grouped, int32_t* cnt,
                              int32_t* scnt, int32_t* sflag) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) {
        const int32_t deg = rp[v + 1] - rp[v];
        const bool big = deg > C;
        int32_t c = big ? (deg + C - 1) / C : 1;
        if (!big && grouped && !group_start(rp, v, C)) c = 0;
        cnt[v] = c;
        scnt[v] = big ? c : 0;
        sflag[v] = big;
    } else if (v == n) {
        cnt[n] = 0;
        scnt[n] = 0;
        sflag[n] = 0;
    }
}

__global__ void k_item_fill(const int32_t* __restrict__ rp, int64_t n, int C, const int32_t* __restrict__ off,
                            const int32_t* __restrict__ soff, const int32_t* __restrict__ sidx, int32_t* item_row,
                            int32_t* item_end, int32_t* item_beg, int32_t* item_ee, int32_t* item_slot,
                            int32_t* split_row, int32_t* split_first) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v > n) return;
    if (v == n) {
        split_first[sidx[n]] = soff[n];
        return;
    }
    const int32_t c = off[v + 1] - off[v];
    if (c == 0) return;  // inside a group that an earlier row starts
    const int32_t b = rp[v], e = rp[v + 1];
    if (e - b > C) {
        for (int32_t j = 0; j < c; ++j) {
            const int32_t i = off[v] + j;
            item_row[i] = (int32_t)v;
            item_end[i] = (int32_t)v + 1;
            item_beg[i] = b + j * C;
            item_ee[i] = min(b + (j + 1) * C, e);
            item_slot[i] = soff[v] + j;
        }
        split_row[sidx[v]] = (int32_t)v;
        split_first[sidx[v]] = soff[v];
        return;
    }
    // the item runs to the next row that starts one (at most 32 rows on)
    int64_t r = v + 1;
    while (r < n && off[r + 1] == off[r]) ++r;
    const int32_t i = off[v];
    item_row[i] = (int32_t)v;
    item_end[i] = (int32_t)r;
    item_beg[i] = b;
    item_ee[i] = rp[r];
    item_slot[i] = -1;
}

int build_items(const CsrView& a, int C, bool grouped, RowItems& it, cudaStream_t s) {
    const int64_t n = a.nrows;
    int32_t *cnt = nullptr, *off = nullptr;
    GBK_CUDA(cudaMallocAsync(&cnt, sizeof(int32_t) * 3 * (n + 1), s));
    GBK_CUDA(cudaMallocAsync(&off, sizeof(int32_t) * 3 * (n + 1), s));
    int32_t *soff = off + (n + 1), *sidx = off + 2 * (n + 1);
    const unsigned g = (unsigned)((n + 1 + 255) / 256);
    k_item_counts<<<g, 256, 0, s>>>(a.ptr, n, C, grouped ? 1 : 0, cnt, cnt + (n + 1), cnt + 2 * (n + 1));
    GBK_LAUNCHED();
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int)(n + 1), s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&tmp, tb, s));
    for (int k = 0; k < 3; ++k) {
        GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt + k * (n + 1), off + k * (n + 1), (int)(n + 1), s));
        count_launch(1);
    }
    int32_t tot[3];
    GBK_CUDA(cudaMemcpyAsync(&tot[0], off + n, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaMemcpyAsync(&tot[1], soff + n, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaMemcpyAsync(&tot[2], sidx + n, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    it.nitems = tot[0];
    it.nslots = tot[1];
    it.nsplit = tot[2];
    const size_t ni = sizeof(int32_t) * std::max<int64_t>(it.nitems, 1);
    GBK_CUDA(cudaMalloc(&it.item_row, ni));
    GBK_CUDA(cudaMalloc(&it.item_end, ni));
    GBK_CUDA(cudaMalloc(&it.item_beg, ni));
    GBK_CUDA(cudaMalloc(&it.item_ee, ni));
    GBK_CUDA(cudaMalloc(&it.item_slot, ni));
    GBK_CUDA(cudaMalloc(&it.split_row, sizeof(int32_t) * std::max<int64_t>(it.nsplit, 1)));
    GBK_CUDA(cudaMalloc(&it.split_first, sizeof(int32_t) * (it.nsplit + 1)));
    k_item_fill<<<g, 256, 0, s>>>(a.ptr, n, C, off, soff, sidx, it.item_row, it.item_end, it.item_beg, it.item_ee,
                                  it.item_slot, it.split_row, it.split_first);
    GBK_LAUNCHED();
    cudaFreeAsync(tmp, s);
    cudaFreeAsync(cnt, s);
    cudaFreeAsync(off, s);
    GBK_CUDA(cudaStreamSynchronize(s));
    return GBK_SUCCESS;
}

// lanes -> rows transpose of a row-interleaved [n][32] store: row j of dst
// receives lane lane_lo + j; `which` (per lane, may be NULL) picks b0 / b1.
template <typename T>
__global__ void k_extract_cols(const T* __restrict__ b0, const T* __restrict__ b1, const int32_t* __restrict__ which,
                               int64_t n, int lane_lo, int nl, T* __restrict__ dst, int64_t stride) {
    __shared__ T tile[32][33];
    const int64_t v0 = (int64_t)blockIdx.x * 32;
    const int k = threadIdx.x;
    const T* src = (which && (which[k] & 1)) ? b1 : b0;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int64_t v = v0 + r;
        if (v < n) tile[r][k] = src[v * 32 + k];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < nl; j += blockDim.y) {
        const int64_t v = v0 + threadIdx.x;
        if (v < n) dst[(int64_t)j * stride + v] = tile[threadIdx.x][lane_lo + j];
    }
}

// Per-lane result summaries; blockIdx.y is the lane.  KIND 0: BFS levels
// in rows of `stride`; 1: PPR ranks [n][32] in b0 / b1 by which[lane];
// 2: SSSP distances [n][32].
template <int KIND>
__global__ void k_digest(const void* __restrict__ b0, const void* __restrict__ b1, const int32_t* __restrict__ which,
                         int64_t n, int64_t stride, unsigned long long mask, LaneDigest* out) {
    const int lane = blockIdx.y;
    if (!((mask >> lane) & 1)) return;
    unsigned long long reached = 0, isum = 0;
    double fsum = 0;
    const float* fb = (KIND == 1 && (which[lane] & 1)) ? (const float*)b1 : (const float*)b0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (KIND == 0) {
            const int32_t x = ((const int32_t*)b0)[(int64_t)lane * stride + v];
            if (x > 0) {
                reached++;
                isum += (unsigned long long)x;
            }
        } else if (KIND == 1) {
            const float x = fb[v * 32 + lane];
            if (x > 0.f) reached++;
            fsum += (double)x;
        } else {
            const int32_t x = ((const int32_t*)b0)[v * 32 + lane];
            if (x != INT_MAX) {
                reached++;
                isum += (unsigned long long)(long long)x;
            }
        }
    }
    reached = warp_sum64(reached);
    isum = warp_sum64(isum);
#pragma unroll
    for (int o = 16; o; o >>= 1) fsum += __shfl_xor_sync(kFull, fsum, o);
    if ((threadIdx.x & 31) == 0) {
        if (reached) atomicAdd((unsigned long long*)&out[lane].reached, reached);
        if (isum) atomicAdd((unsigned long long*)&out[lane].isum, isum);
        if (fsum != 0.0) atomicAdd(&out[lane].fsum, fsum);
    }
}

template <int KIND>
int launch_digest(const void* b0, const void* b1, const int32_t* which, int64_t n, int64_t stride,
                  unsigned long long mask, int lanes, LaneDigest* out, cudaStream_t s) {
    GBK_CUDA(cudaMemsetAsync(out, 0, sizeof(LaneDigest) * lanes, s));
    if (!mask || n == 0) return GBK_SUCCESS;
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 2));
    k_digest<KIND><<<dim3(gx, lanes), 256, 0, s>>>(b0, b1, which, n, stride, mask, out);
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

struct Lanes64 {
    int32_t v[64];
};
struct Lanes32 {
    int32_t v[32];
};

template <typename S>
__global__ void k_set_launch(S* st, int budget, int stop_on_finish) {
    st->launch_budget = budget;
    st->stop_on_finish = stop_on_finish;
    st->st.launch_iters = 0;
}

// ============================================================================
// 64-lane BFS

struct BfsCfg {
    const int32_t* rp;
    const int32_t* col;
    const int32_t* cp;
    const int32_t* row;
    int64_t n, nnz;
    unsigned long long* visited;
    unsigned long long* buf[2];
    int32_t* levels;
    int64_t stride;
    int2* chunks;      // top-down: 256-entry pieces of rows longer than 32 entries, (vertex, first entry)
    int32_t* nchunks;  // pieces appended this iteration
};

struct BfsState {
    BatchStatus st;
    unsigned long long alive, m_front, m_unvis, n_front;
    unsigned long long last_m_front, last_m_unvis, last_n_front;
    int32_t launch_budget, stop_on_finish, pull, dir_mode, alpha, beta;
};

__device__ __forceinline__ int bfs_pick_pull(const BfsState* st, int cur_pull, int64_t n) {
    if (st->dir_mode == 1) return 0;
    if (st->dir_mode == 2) return 1;
    if (!cur_pull) return st->last_m_front * (unsigned long long)st->alpha > st->last_m_unvis ? 1 : 0;
    return st->last_n_front * (unsigned long long)st->beta < (unsigned long long)n ? 0 : 1;
}

// Top-down step: each frontier vertex ORs its lane word into the next word
// of every out-neighbour that some of those lanes have not visited.  Short
// rows are walked by one thread; rows of more than 32 entries are cut into
// 256-entry pieces that k_bfs_push_pieces hands out one per warp (a hub row
// of 10^4 - 10^5 entries on one warp held the whole iteration back).
__global__ void __launch_bounds__(kBT) k_bfs_push(const BfsCfg* __restrict__ cfg, const BfsState* __restrict__ st) {
    if (st->pull || st->st.active == 0) return;
    const int64_t n = cfg->n;
    const int32_t* __restrict__ rp = cfg->rp;
    const int32_t* __restrict__ col = cfg->col;
    const int it = st->st.iter;
    const unsigned long long* __restrict__ fr = cfg->buf[it & 1];
    unsigned long long* nx = cfg->buf[(it + 1) & 1];
    const unsigned long long* __restrict__ vis = cfg->visited;
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kBT) >> 5;
    for (int64_t base = wid * 32; base < n; base += nwarps * 32) {
        const int64_t v = base + lane;
        unsigned long long f = 0;
        int32_t b = 0, e = 0;
        if (v < n) {
            f = fr[v];
            if (f) {
                b = rp[v];
                e = rp[v + 1];
            }
        }
        const bool big = f && (e - b) > 32;
        if (f && !big) {
            for (int32_t k = b; k < e; ++k) {
                const int32_t u = col[k];
                const unsigned long long m = f & ~vis[u];
                if (m) atomicOr(nx + u, m);
            }
        }
        // long rows: append their pieces, one atomic per warp
        const int32_t np = big ? (e - b + kBfsPiece - 1) / kBfsPiece : 0;
        int32_t incl = np;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        const int32_t total = __shfl_sync(kFull, incl, 31);
        if (total) {
            int32_t base0 = 0;
            if (lane == 0) base0 = atomicAdd(cfg->nchunks, total);
            base0 = __shfl_sync(kFull, base0, 0);
            for (int32_t i = 0; i < np; ++i)
                cfg->chunks[base0 + incl - np + i] = make_int2((int32_t)v, b + i * kBfsPiece);
        }
    }
}

// The pieces k_bfs_push appended, one warp per piece.
__global__ void __launch_bounds__(kBT) k_bfs_push_pieces(const BfsCfg* __restrict__ cfg,
                                                         const BfsState* __restrict__ st) {
    if (st->pull || st->st.active == 0) return;
    const int32_t np = *cfg->nchunks;
    const int32_t* __restrict__ rp = cfg->rp;
    const int32_t* __restrict__ col = cfg->col;
    const int it = st->st.iter;
    const unsigned long long* __restrict__ fr = cfg->buf[it & 1];
    unsigned long long* nx = cfg->buf[(it + 1) & 1];
    const unsigned long long* __restrict__ vis = cfg->visited;
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kBT) >> 5;
    for (int64_t c = wid; c < np; c += nwarps) {
        const int2 pc = cfg->chunks[c];
        const unsigned long long ff = fr[pc.x];
        const int32_t ee = min(pc.y + kBfsPiece, rp[pc.x + 1]);
        for (int32_t k = pc.y + lane; k < ee; k += 32) {
            const int32_t u = col[k];
            const unsigned long long m = ff & ~vis[u];
            if (m) atomicOr(nx + u, m);
        }
    }
}

// Bottom-up step: each vertex with unvisited active lanes ORs the frontier
// words of its in-neighbours (CSC row) and stops once every such lane is found.
__global__ void __launch_bounds__(kBT) k_bfs_pull(const BfsCfg* __restrict__ cfg, const BfsState* __restrict__ st) {
    if (!st->pull || st->st.active == 0) return;
    const unsigned long long act = st->st.active;
    const int64_t n = cfg->n;
    const int32_t* __restrict__ cp = cfg->cp;
    const int32_t* __restrict__ row = cfg->row;
    const int it = st->st.iter;
    const unsigned long long* __restrict__ fr = cfg->buf[it & 1];
    unsigned long long* nx = cfg->buf[(it + 1) & 1];
    const unsigned long long* __restrict__ vis = cfg->visited;
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kBT) >> 5;
    for (int64_t base = wid * 32; base < n; base += nwarps * 32) {
        const int64_t v = base + lane;
        unsigned long long un = 0;
        int32_t b = 0, e = 0;
        if (v < n) {
            un = ~vis[v] & act;
            if (un) {
                b = cp[v];
                e = cp[v + 1];
            }
        }
        const bool big = un && (e - b) > 32;
        if (un && !big) {
            unsigned long long acc = 0;
            for (int32_t k = b; k < e; ++k) {
                acc |= fr[row[k]];
                if ((acc & un) == un) break;
            }
            acc &= un;
            if (acc) nx[v] = acc;
        }
        unsigned bigm = __ballot_sync(kFull, big);
        while (bigm) {
            const int src = __ffs(bigm) - 1;
            bigm &= bigm - 1;
            const unsigned long long uu = __shfl_sync(kFull, un, src);
            const int32_t bb = __shfl_sync(kFull, b, src), ee = __shfl_sync(kFull, e, src);
            unsigned long long acc = 0;
            for (int32_t k0 = bb; k0 < ee; k0 += 32) {
                const int32_t k = k0 + lane;
                const unsigned long long x = k < ee ? fr[row[k]] : 0ull;
                acc |= warp_or64(x);
                if ((acc & uu) == uu) break;
            }
            acc &= uu;
            if (lane == 0 && acc) nx[base + src] = acc;
        }
    }
}

// Keeps the new bits that were not visited, marks them visited, writes their
// levels, clears the consumed frontier and gathers the direction statistics.
__global__ void __launch_bounds__(kBT) k_bfs_finalize(const BfsCfg* __restrict__ cfg, BfsState* st) {
    __shared__ int32_t depth[64];
    __shared__ unsigned long long s_alive, s_mf, s_mu, s_nf;
    if (threadIdx.x < 64) depth[threadIdx.x] = st->st.iters[threadIdx.x] + 1;
    if (threadIdx.x == 0) s_alive = s_mf = s_mu = s_nf = 0;
    __syncthreads();
    const unsigned long long act = st->st.active;
    const int64_t n = cfg->n;
    const int it = st->st.iter;
    unsigned long long* fr = cfg->buf[it & 1];
    unsigned long long* nx = cfg->buf[(it + 1) & 1];
    unsigned long long* visited = cfg->visited;
    const int32_t* __restrict__ rp = cfg->rp;
    int32_t* levels = cfg->levels;
    const int64_t stride = cfg->stride;
    unsigned long long alive = 0, mf = 0, mu = 0, nf = 0;
    if (act) {
        for (int64_t v = (int64_t)blockIdx.x * kBT + threadIdx.x; v < n; v += (int64_t)gridDim.x * kBT) {
            if (fr[v]) fr[v] = 0;
            const unsigned long long x = nx[v];
            unsigned long long vis = visited[v];
            const unsigned long long nw = x & ~vis & act;
            if (x != nw) nx[v] = nw;
            const unsigned long long deg = (unsigned long long)(rp[v + 1] - rp[v]);
            if (nw) {
                vis |= nw;
                visited[v] = vis;
                alive |= nw;
                mf += deg;
                nf += 1;
                unsigned long long bits = nw;
                while (bits) {
                    const int s = __ffsll((long long)bits) - 1;
                    bits &= bits - 1;
                    levels[(int64_t)s * stride + v] = depth[s];
                }
            }
            if (~vis & act) mu += deg;
        }
    }
    alive = warp_or64(alive);
    mf = warp_sum64(mf);
    mu = warp_sum64(mu);
    nf = warp_sum64(nf);
    if ((threadIdx.x & 31) == 0) {
        if (alive) atomicOr(&s_alive, alive);
        if (mf) atomicAdd(&s_mf, mf);
        if (mu) atomicAdd(&s_mu, mu);
        if (nf) atomicAdd(&s_nf, nf);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_alive) atomicOr(&st->alive, s_alive);
        if (s_mf) atomicAdd(&st->m_front, s_mf);
        if (s_mu) atomicAdd(&st->m_unvis, s_mu);
        if (s_nf) atomicAdd(&st->n_front, s_nf);
    }
}

__global__ void k_bfs_control(BfsState* st, int64_t n, int32_t* nchunks, cudaGraphConditionalHandle h) {
    const int s = threadIdx.x;
    const unsigned long long act = st->st.active, alive = st->alive;
    if (s < 64 && ((act >> s) & 1) && ((alive >> s) & 1)) st->st.iters[s] += 1;
    __syncthreads();
    if (s == 0) {
        const unsigned long long fin = act & ~alive;
        st->st.active = act & alive;
        st->st.finished |= fin;
        st->st.iter += 1;
        st->st.launch_iters += 1;
        st->last_m_front = st->m_front;
        st->last_m_unvis = st->m_unvis;
        st->last_n_front = st->n_front;
        st->pull = bfs_pick_pull(st, st->pull, n);
        st->alive = st->m_front = st->m_unvis = st->n_front = 0;
        *nchunks = 0;
        const bool cont = st->st.active != 0 && st->st.launch_iters < st->launch_budget &&
                          !(st->stop_on_finish && fin);
        if (h) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

__global__ void k_bfs_admit(const BfsCfg* __restrict__ cfg, BfsState* st, unsigned long long mask, Lanes64 src) {
    const int s = threadIdx.x;
    if (s < 64 && ((mask >> s) & 1)) {
        const int32_t v = src.v[s];
        const unsigned long long bit = 1ull << s;
        atomicOr(cfg->visited + v, bit);
        atomicOr(cfg->buf[st->st.iter & 1] + v, bit);
        cfg->levels[(int64_t)s * cfg->stride + v] = 1;
        st->st.iters[s] = 1;
        atomicAdd(&st->last_m_front, (unsigned long long)(cfg->rp[v + 1] - cfg->rp[v]));
        atomicAdd(&st->last_n_front, 1ull);
    }
    __syncthreads();
    if (s == 0) {
        st->st.active |= mask;
        st->st.finished &= ~mask;
        // every vertex is unvisited for the new lanes
        st->last_m_unvis = (unsigned long long)cfg->nnz;
        st->pull = bfs_pick_pull(st, 0, cfg->n);
    }
}

__global__ void k_bfs_release(const BfsCfg* __restrict__ cfg, BfsState* st, unsigned long long mask) {
    const int64_t n = cfg->n;
    unsigned long long* visited = cfg->visited;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long x = visited[v];
        if (x & mask) visited[v] = x & ~mask;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->st.finished &= ~mask;
}

__global__ void k_bfs_set_mode(BfsState* st, int dir_mode, int alpha, int beta) {
    st->dir_mode = dir_mode;
    st->alpha = alpha;
    st->beta = beta;
}

struct BfsBatch final : Batch {
    gbk_matrix A = nullptr;
    BfsCfg cfg{};
    BfsCfg* d_cfg = nullptr;
    BfsState* d_st = nullptr;
    BatchStatus* h_st = nullptr;
    int32_t* own_levels = nullptr;  // [64][n], allocated on the first admission into it
    LoopGraph loop;
    int grid_push = 0, grid_pieces = 0, grid_pull = 0, grid_fin = 0;
    size_t bytes = 0;

    ~BfsBatch() override {
        cudaFree(cfg.visited);
        cudaFree(cfg.buf[0]);
        cudaFree(cfg.nchunks);
        cudaFree(own_levels);
        cudaFree(d_cfg);
        cudaFree(d_st);
        cudaFreeHost(h_st);
    }
    int kind() const override { return kBatchBfs; }
    int lanes() const override { return kBfsLanes; }
    const BatchStatus* host() const override { return h_st; }
    size_t device_bytes() const override { return bytes; }
    size_t lane_bytes() const override { return (size_t)cfg.n * 4; }
    int kernels_per_iter() const override { return 5; }

    int init(gbk_matrix a, const BatchOptions& o, cudaStream_t s) {
        A = a;
        int rc = ensure_csc(A, s);
        if (rc) return rc;
        const int64_t n = A->csr.nrows;
        cfg.rp = A->csr.ptr;
        cfg.col = A->csr.idx;
        cfg.cp = A->csc.ptr;
        cfg.row = A->csc.idx;
        cfg.n = n;
        cfg.nnz = A->csr.nnz;
        const size_t words = (size_t)std::max<int64_t>(n, 1);
        GBK_CUDA(cudaMalloc(&cfg.visited, 8 * words));
        GBK_CUDA(cudaMalloc(&cfg.buf[0], 16 * words));
        cfg.buf[1] = cfg.buf[0] + words;
        cfg.levels = nullptr;
        cfg.stride = n;
        GBK_CUDA(cudaMemsetAsync(cfg.visited, 0, 8 * words, s));
        GBK_CUDA(cudaMemsetAsync(cfg.buf[0], 0, 16 * words, s));
        // every vertex is in the frontier once per iteration, and a row of d > 32
        // entries gives ceil(d / 256) <= d / 32 pieces: nnz / 32 + 1 bound them
        const size_t npieces = (size_t)(A->csr.nnz / 32 + 1);
        GBK_CUDA(cudaMalloc(&cfg.nchunks, 16 + sizeof(int2) * npieces));
        GBK_CUDA(cudaMemsetAsync(cfg.nchunks, 0, 16, s));
        cfg.chunks = reinterpret_cast<int2*>(reinterpret_cast<char*>(cfg.nchunks) + 16);
        GBK_CUDA(cudaMalloc(&d_cfg, sizeof(BfsCfg)));
        GBK_CUDA(cudaMalloc(&d_st, sizeof(BfsState)));
        GBK_CUDA(cudaMallocHost(&h_st, sizeof(BatchStatus)));
        memset(h_st, 0, sizeof(BatchStatus));
        GBK_CUDA(cudaMemcpyAsync(d_cfg, &cfg, sizeof(BfsCfg), cudaMemcpyHostToDevice, s));
        BfsState init{};
        init.dir_mode = o.bfs_direction;
        init.alpha = o.bfs_alpha;
        init.beta = o.bfs_beta;
        init.launch_budget = 1;
        GBK_CUDA(cudaMemcpyAsync(d_st, &init, sizeof(BfsState), cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        bytes = 8 * words * 3 + 16 + sizeof(int2) * npieces;
        grid_push = persistent_blocks((const void*)k_bfs_push, kBT);
        grid_pieces = persistent_blocks((const void*)k_bfs_push_pieces, kBT);
        grid_pull = persistent_blocks((const void*)k_bfs_pull, kBT);
        grid_fin = persistent_blocks((const void*)k_bfs_finalize, kBT);
        return build_loop(loop, [this, n](cudaStream_t cs, cudaGraphConditionalHandle h) -> int {
            k_bfs_push<<<grid_push, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_bfs_push_pieces<<<grid_pieces, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_bfs_pull<<<grid_pull, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_bfs_finalize<<<grid_fin, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_bfs_control<<<1, 64, 0, cs>>>(d_st, n, cfg.nchunks, h);
            GBK_LAUNCH_CHECK();
            return GBK_SUCCESS;
        });
    }

    // levels == NULL returns to the batch's own lane rows.
    int set_levels(int32_t* levels, int64_t stride, cudaStream_t s) {
        cfg.levels = levels ? levels : own_levels;
        cfg.stride = levels ? stride : cfg.n;
        GBK_CUDA(cudaMemcpyAsync(d_cfg, &cfg, sizeof(BfsCfg), cudaMemcpyHostToDevice, s));
        return GBK_SUCCESS;
    }

    int set_mode(int dir_mode, int alpha, int beta, cudaStream_t s) {
        k_bfs_set_mode<<<1, 1, 0, s>>>(d_st, dir_mode, alpha, beta);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }

    int admit(unsigned long long mask, const int32_t* src, cudaStream_t s) override {
        if (!mask) return GBK_SUCCESS;
        if (!cfg.levels) {
            const size_t row = 4 * (size_t)std::max<int64_t>(cfg.n, 1);
            GBK_CUDA(cudaMalloc(&own_levels, row * kBfsLanes));
            bytes += row * kBfsLanes;
            const int rc = set_levels(nullptr, 0, s);
            if (rc) return rc;
        }
        Lanes64 l{};
        for (int k = 0; k < kBfsLanes; ++k)
            if ((mask >> k) & 1) {
                GBK_REQUIRE(src[k] >= 0 && src[k] < cfg.n, GBK_INVALID_INDEX,
                            "batched BFS: source %d out of range [0, %lld)", src[k], (long long)cfg.n);
                l.v[k] = src[k];
                GBK_CUDA(cudaMemsetAsync(cfg.levels + (int64_t)k * cfg.stride, 0, 4 * (size_t)cfg.n, s));
            }
        k_bfs_admit<<<1, 64, 0, s>>>(d_cfg, d_st, mask, l);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }

    int launch(int budget, bool stop_on_finish, cudaStream_t s) override {
        k_set_launch<BfsState><<<1, 1, 0, s>>>(d_st, budget, stop_on_finish ? 1 : 0);
        GBK_LAUNCHED();
        return run_loop(loop, &d_st->st, h_st, budget, stop_on_finish, s);
    }

    int extract(int lane_lo, int nl, void* dst, int64_t stride, cudaStream_t s) override {
        GBK_REQUIRE(lane_lo >= 0 && nl >= 0 && lane_lo + nl <= kBfsLanes, GBK_INVALID_INDEX, "BFS extract: bad lanes");
        GBK_REQUIRE(nl == 0 || cfg.levels, GBK_INVALID_OBJECT, "BFS extract: no lane has run yet");
        for (int j = 0; j < nl; ++j)
            GBK_CUDA(cudaMemcpyAsync((int32_t*)dst + (int64_t)j * stride,
                                     cfg.levels + (int64_t)(lane_lo + j) * cfg.stride, 4 * (size_t)cfg.n,
                                     cudaMemcpyDefault, s));
        return GBK_SUCCESS;
    }

    int digest(unsigned long long mask, LaneDigest* d_out, cudaStream_t s) override {
        GBK_REQUIRE(!mask || cfg.levels, GBK_INVALID_OBJECT, "BFS digest: no lane has run yet");
        return launch_digest<0>(cfg.levels, nullptr, nullptr, cfg.n, cfg.stride, mask, kBfsLanes, d_out, s);
    }

    int release(unsigned long long mask, cudaStream_t s) override {
        if (!mask) return GBK_SUCCESS;
        k_bfs_release<<<grid_fin, kBT, 0, s>>>(d_cfg, d_st, mask);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }
};

// ============================================================================
// column-lane batches (PPR and SSSP share the work items and this config)

struct ColCfg {
    const int32_t* rp;
    const int32_t* col;
    const void* val;
    int vtype;
    int item_edges;
    int64_t n, nnz;
    const int32_t* item_row;
    const int32_t* item_end;
    const int32_t* item_beg;
    const int32_t* item_ee;
    const int32_t* item_slot;
    int64_t nitems;
    const int32_t* split_row;
    const int32_t* split_first;
    int64_t nsplit;
    // PPR
    const int32_t* cdeg;
    const float* d;
    float* r[2];
    float* w[2];
    float* split_acc;
    double* partial;  // [parts][2][32]
    int32_t parts_main;  // blocks of k_ppr_update, one partial each
    // SSSP
    int32_t* dist;
    uint32_t* chg[2];
};

// ----------------------------------------------------------------------------
// 32-column personalised PageRank (plus-second SpMM with a fused epilogue)

struct PprState {
    BatchStatus st;
    int32_t seed[32];
    float tele[32];
    float rdiff[32];
    int32_t result_buf[32];
    int32_t launch_budget, stop_on_finish, itermax, pad;
    double damping, tol;
};

// The SpMM leaves each non-empty row's sum for the active lanes in r_out;
// k_ppr_update turns it into the new rank.  Lane q of a quarter-warp holds
// columns 4q .. 4q + 3; only the active ones are stored.
__device__ __forceinline__ void ppr_store_sum4(float* r_out, int64_t row, float4 s, unsigned m4, int q) {
    float* p = r_out + row * 32 + 4 * q;
    if (m4 == 0xFu) {
        __stcs(reinterpret_cast<float4*>(p), s);
        return;
    }
    if (m4 & 1u) __stcs(p, s.x);
    if (m4 & 2u) __stcs(p + 1, s.y);
    if (m4 & 4u) __stcs(p + 2, s.z);
    if (m4 & 8u) __stcs(p + 3, s.w);
}

__device__ __forceinline__ float4 ld_keep4(const float* p, uint64_t pol) {
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// (quarter 0 + quarter 1) + (quarter 2 + quarter 3), on every lane: float
// addition commutes, so all four quarters end with the same bits.
__device__ __forceinline__ float4 quarter_sum4(float4 a) {
#pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
        a.x += __shfl_xor_sync(kFull, a.x, o);
        a.y += __shfl_xor_sync(kFull, a.y, o);
        a.z += __shfl_xor_sync(kFull, a.z, o);
        a.w += __shfl_xor_sync(kFull, a.w, o);
    }
    return a;
}

// 4-edge blocks each warp keeps in flight: 16 gathered 128-byte w rows.
constexpr int kPprBlocks = 4;

// One warp per work item.  An item is either a run of up to 32 consecutive
// short rows or one piece of a long row.  The warp loads 32 column ids at a
// time and works on 4 edges at once: quarter g (lanes 8g .. 8g + 7) gathers
// the 128-byte w row of the item's edges g, g + 4, g + 8, ... as one 16-byte
// load per lane (lane q: columns 4q .. 4q + 3).  Each quarter sums its edges of
// a row in CSR order; when the edge index passes the row's end the quarters'
// sums are added in a fixed order and stored.  The order of every column's
// sum depends on the graph and the item cut only, never on which other
// columns are active.  Lanes whose four columns are all inactive issue no
// loads.  Pieces of split rows park their sums for k_ppr_fix.
__global__ void __launch_bounds__(kBT, 4) k_ppr_spmm(const ColCfg* __restrict__ cfg, const PprState* __restrict__ st) {
    const unsigned act = (unsigned)st->st.active;
    if (!act) return;
    const int lane = threadIdx.x & 31, g = lane >> 3, q = lane & 7;
    const unsigned m4 = (act >> (4 * q)) & 0xFu;
    const bool any = m4 != 0;
    const int cur = st->st.iter & 1;
    const float* __restrict__ w_q = cfg->w[cur] + 4 * q;
    float* r_out = cfg->r[cur ^ 1];
    const int32_t* __restrict__ rp = cfg->rp;
    const int32_t* __restrict__ col = cfg->col;
    const uint64_t pol = policy_evict_last();
    const int64_t nitems = cfg->nitems;
    const int64_t gw = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kBT) >> 5;
    for (int64_t it = gw; it < nitems; it += nw) {
        int32_t row = cfg->item_row[it];
        const int32_t row0 = row, row_end = cfg->item_end[it];
        const int32_t eb = cfg->item_beg[it], ee = cfg->item_ee[it];
        const int32_t slot = cfg->item_slot[it];
        // the ends of the item's rows (at most 32), one per lane: row r ends
        // at lane r - row0's value (a split piece ends at its own end)
        const int32_t rpl = (slot < 0 && row0 + 1 + lane <= row_end) ? rp[row0 + 1 + lane] : ee;
        int32_t bound = __shfl_sync(kFull, rpl, 0);
        int32_t start = eb;  // where the current row begins
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int32_t e0 = eb; e0 < ee; e0 += 32) {
            const int cnt = min(32, ee - e0);
            const int32_t cl = lane < cnt ? __ldcs(col + e0 + lane) : 0;
            for (int j = 0; j < cnt; j += 4 * kPprBlocks) {
                float4 t[kPprBlocks];
#pragma unroll
                for (int b = 0; b < kPprBlocks; ++b) {
                    const int k = j + 4 * b + g;
                    const int32_t u = __shfl_sync(kFull, cl, k & 31);
                    t[b] = (any && k < cnt) ? ld_keep4(w_q + ((int64_t)u << 5), pol) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                // all these edges inside the current row: plain adds (edges
                // past cnt were loaded as +0, which leaves the sums unchanged)
                if (e0 + min(j + 4 * kPprBlocks, cnt) <= bound) {
#pragma unroll
                    for (int b = 0; b < kPprBlocks; ++b) acc = add4(acc, t[b]);
                    continue;
                }
#pragma unroll
                for (int b = 0; b < kPprBlocks; ++b) {
                    const int nb = min(4, cnt - (j + 4 * b));  // edges of this block (warp-uniform)
                    if (nb <= 0) break;
                    const int32_t base = e0 + j + 4 * b;
                    bool pending = g < nb;
                    while (base + nb > bound) {  // rows that end inside this block (empty rows need no store)
                        if (pending && base + g < bound) {
                            acc = add4(acc, t[b]);
                            pending = false;
                        }
                        const float4 s = quarter_sum4(acc);
                        if (g == 0 && bound > start) ppr_store_sum4(r_out, row, s, m4, q);
                        acc = make_float4(0.f, 0.f, 0.f, 0.f);
                        start = bound;
                        ++row;
                        bound = __shfl_sync(kFull, rpl, (row - row0) & 31);
                    }
                    if (pending) acc = add4(acc, t[b]);
                }
            }
        }
        const float4 s = quarter_sum4(acc);
        if (slot >= 0) {
            if (g == 0) *reinterpret_cast<float4*>(cfg->split_acc + (int64_t)slot * 32 + 4 * q) = s;
            continue;
        }
        if (g == 0 && row < row_end && bound > start) ppr_store_sum4(r_out, row, s, m4, q);
    }
}

// Lane k stores column k of a split row's sum.
__device__ __forceinline__ void ppr_store_sum(float* r_out, int64_t row, float acc, bool mine) {
    if (mine) __stcs(r_out + row * 32 + (threadIdx.x & 31), acc);
}

__global__ void __launch_bounds__(kBT) k_ppr_fix(const ColCfg* __restrict__ cfg, const PprState* __restrict__ st) {
    const unsigned act = (unsigned)st->st.active;
    if (!act) return;
    const int lane = threadIdx.x & 31;
    float* r_out = cfg->r[(st->st.iter & 1) ^ 1];
    const bool mine = (act >> lane) & 1;
    const int64_t gw = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kBT) >> 5;
    for (int64_t i = gw; i < cfg->nsplit; i += nw) {
        // four independent partial sums (slots k mod 4), added in a fixed order
        float a[4] = {0.f, 0.f, 0.f, 0.f};
        const int32_t s0 = cfg->split_first[i], s1 = cfg->split_first[i + 1];
        int32_t sl = s0;
        for (; sl + 4 <= s1; sl += 4) {
#pragma unroll
            for (int k = 0; k < 4; ++k) a[k] += cfg->split_acc[(int64_t)(sl + k) * 32 + lane];
        }
        for (int k = 0; sl < s1; ++sl, ++k) a[k] += cfg->split_acc[(int64_t)sl * 32 + lane];
        ppr_store_sum(r_out, cfg->split_row[i], (a[0] + a[1]) + (a[2] + a[3]), mine);
    }
}

// Elementwise step over all n x 32 entries, as float4 (thread t always on
// columns 4 (t % 8) .. 4 (t % 8) + 3): rank = row sum (0 for empty rows) plus
// the teleport at the seed, w = rank / d, and the per-column partial sums of
// |rank - old| and of the rank held by sinks, per block in a fixed order.
// Inactive columns are written back unchanged.
__global__ void __launch_bounds__(kBT, 3) k_ppr_update(const ColCfg* __restrict__ cfg, const PprState* __restrict__ st) {
    __shared__ double s_sink[kBT / 32][32], s_rd[kBT / 32][32];
    const unsigned act = (unsigned)st->st.active;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, quad = threadIdx.x & 7;
    double sink[4] = {0, 0, 0, 0}, rd[4] = {0, 0, 0, 0};
    if (act) {
        bool m[4];
        int32_t seed[4];
        float tele[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            m[c] = (act >> (4 * quad + c)) & 1;
            seed[c] = st->seed[4 * quad + c];
            tele[c] = st->tele[4 * quad + c];
        }
        const int cur = st->st.iter & 1;
        const float4* __restrict__ r_old = (const float4*)cfg->r[cur];
        float4* r_out = (float4*)cfg->r[cur ^ 1];
        float4* w_out = (float4*)cfg->w[cur ^ 1];
        const int32_t* __restrict__ rp = cfg->rp;
        const int64_t total = cfg->n * 8;
        const int64_t stride = (int64_t)gridDim.x * kBT;
        constexpr int U = 2;
        for (int64_t i0 = (int64_t)blockIdx.x * kBT + threadIdx.x; i0 < total; i0 += U * stride) {
            float4 acc[U], old[U];
            float dv[U];
            int32_t cd[U];
            bool ne[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int64_t i = i0 + k * stride;
                if (i < total) {
                    const int64_t v = i >> 3;
                    ne[k] = rp[v + 1] > rp[v];
                    acc[k] = __ldcs(r_out + i);
                    old[k] = __ldcs(r_old + i);
                    dv[k] = cfg->d[v];
                    cd[k] = cfg->cdeg[v];
                }
            }
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int64_t i = i0 + k * stride;
                if (i >= total) continue;
                const int64_t v = i >> 3;
                float a[4] = {acc[k].x, acc[k].y, acc[k].z, acc[k].w};
                const float o[4] = {old[k].x, old[k].y, old[k].z, old[k].w};
                float wv[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    if (m[c]) {
                        const float x = ne[k] ? a[c] : 0.f;
                        const float rn = (v == seed[c]) ? tele[c] + x : x;
                        a[c] = rn;
                        rd[c] += (double)fabsf(o[c] - rn);
                        if (cd[k] == 0) sink[c] += (double)rn;
                    }
                    wv[c] = a[c] / dv[k];
                }
                __stcs(r_out + i, make_float4(a[0], a[1], a[2], a[3]));
                __stcs(w_out + i, make_float4(wv[0], wv[1], wv[2], wv[3]));
            }
        }
    }
    // lanes l, l + 8, l + 16, l + 24 hold the same columns
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        for (int o = 8; o < 32; o <<= 1) {
            sink[c] += __shfl_xor_sync(kFull, sink[c], o);
            rd[c] += __shfl_xor_sync(kFull, rd[c], o);
        }
    }
    if (lane < 8) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            s_sink[warp][4 * lane + c] = sink[c];
            s_rd[warp][4 * lane + c] = rd[c];
        }
    }
    __syncthreads();
    if (warp == 0) {
        double x = 0, y = 0;
        for (int w2 = 0; w2 < kBT / 32; ++w2) {
            x += s_sink[w2][lane];
            y += s_rd[w2][lane];
        }
        double* out = cfg->partial + (int64_t)blockIdx.x * 64;
        out[lane] = x;
        out[32 + lane] = y;
    }
}

// 1024 threads: thread (g, k) sums the parts g, g + 32, ... of column k, then
// warp 0 adds the 32 group sums in order (a fixed order: deterministic).
__global__ void __launch_bounds__(1024) k_ppr_control(const ColCfg* __restrict__ cfg, PprState* st,
                                                      cudaGraphConditionalHandle h) {
    __shared__ double s_sink[32][33], s_rd[32][33];
    const int k = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const int parts = cfg->parts_main;
    double sink = 0, rd = 0;
    for (int p = grp; p < parts; p += 32) {
        sink += cfg->partial[(int64_t)p * 64 + k];
        rd += cfg->partial[(int64_t)p * 64 + 32 + k];
    }
    s_sink[grp][k] = sink;
    s_rd[grp][k] = rd;
    __syncthreads();
    if (grp != 0) return;
    sink = 0;
    rd = 0;
    for (int g2 = 0; g2 < 32; ++g2) {
        sink += s_sink[g2][k];
        rd += s_rd[g2][k];
    }
    const unsigned act = (unsigned)st->st.active;
    const int cur = st->st.iter & 1;
    unsigned fin = 0;
    if ((act >> k) & 1) {
        st->st.iters[k] += 1;
        st->rdiff[k] = (float)rd;
        if ((st->tol > 0 && rd < st->tol) || st->st.iters[k] >= st->itermax) {
            fin = 1u << k;
            st->result_buf[k] = cur ^ 1;
        } else {
            st->tele[k] = (float)((1.0 - st->damping) + st->damping * sink);
        }
    }
    fin = __reduce_or_sync(kFull, fin);
    if (k == 0) {
        st->st.active = act & ~fin;
        st->st.finished |= fin;
        st->st.iter += 1;
        st->st.launch_iters += 1;
        const bool cont = st->st.active != 0 && st->st.launch_iters < st->launch_budget &&
                          !(st->stop_on_finish && fin);
        if (h) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// New columns start from r = e_seed, w = r / d.  Only the new lanes are
// touched: thread i covers row i / nl and lane lanes[i % nl].
__global__ void k_ppr_init_cols(const ColCfg* __restrict__ cfg, const PprState* __restrict__ st, Lanes32 lanes,
                                int nl, Lanes32 seeds) {
    const int cur = st->st.iter & 1;
    float* r = cfg->r[cur];
    float* w = cfg->w[cur];
    const int64_t total = cfg->n * nl;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i / nl;
        const int k = lanes.v[i - v * nl];
        const float x = (v == seeds.v[k]) ? 1.0f : 0.0f;
        r[v * 32 + k] = x;
        w[v * 32 + k] = x / cfg->d[v];
    }
}

__global__ void k_ppr_admit(const ColCfg* __restrict__ cfg, PprState* st, unsigned mask, Lanes32 seeds,
                            double damping, double tol, int itermax) {
    const int k = threadIdx.x;
    if (k == 0) {
        st->damping = damping;
        st->tol = tol;
        st->itermax = itermax;
    }
    if ((mask >> k) & 1) {
        const int32_t s = seeds.v[k];
        st->seed[k] = s;
        st->st.iters[k] = 0;
        st->result_buf[k] = -1;
        const double sink0 = cfg->cdeg[s] == 0 ? 1.0 : 0.0;
        st->tele[k] = (float)((1.0 - damping) + damping * sink0);
    }
    __syncwarp();
    if (k == 0) {
        st->st.active |= mask;
        st->st.finished &= ~(unsigned long long)mask;
    }
}

__global__ void k_cols_release(BatchStatus* st, unsigned long long mask) { st->finished &= ~mask; }

__global__ void k_ppr_degree(const int32_t* __restrict__ cp, int64_t n, float damping, int32_t* cdeg, float* d) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int32_t c = cp[v + 1] - cp[v];
    cdeg[v] = c;
    // d = max(d_out / damping, 1 / damping) in FP32 as the reference forms it (pr.hpp:84-90)
    const float a = (float)c / damping, b = 1.0f / damping;
    d[v] = a > b ? a : b;
}

// shared set-up of the column-lane batches
int init_col_cfg(gbk_matrix A, const BatchOptions& o, bool grouped, ColCfg& cfg, RowItems& items,
                 cudaStream_t s) {
    const CsrView& a = A->csr;
    GBK_REQUIRE(a.nrows == a.ncols, GBK_DIMENSION_MISMATCH, "batched traversal: matrix must be square");
    GBK_REQUIRE(o.item_edges >= 32 && o.item_edges % 32 == 0 && o.item_edges <= (1 << 20), GBK_INVALID_VALUE,
                "batched traversal: item_edges must be a multiple of 32 in [32, 2^20]");
    int rc = build_items(a, o.item_edges, grouped, items, s);
    if (rc) return rc;
    cfg.rp = a.ptr;
    cfg.col = a.idx;
    cfg.val = a.val;
    cfg.vtype = A->vtype;
    cfg.item_edges = o.item_edges;
    cfg.n = a.nrows;
    cfg.nnz = a.nnz;
    cfg.item_row = items.item_row;
    cfg.item_end = items.item_end;
    cfg.item_beg = items.item_beg;
    cfg.item_ee = items.item_ee;
    cfg.item_slot = items.item_slot;
    cfg.nitems = items.nitems;
    cfg.split_row = items.split_row;
    cfg.split_first = items.split_first;
    cfg.nsplit = items.nsplit;
    return GBK_SUCCESS;
}

struct PprBatch final : Batch {
    gbk_matrix A = nullptr;
    BatchOptions opt;
    ColCfg cfg{};
    RowItems items;
    ColCfg* d_cfg = nullptr;
    PprState* d_st = nullptr;
    BatchStatus* h_st = nullptr;
    LoopGraph loop;
    int grid_main = 0, grid_fix = 0, grid_upd = 0;
    size_t bytes = 0;

    ~PprBatch() override {
        items.release();
        cudaFree((void*)cfg.cdeg);
        cudaFree((void*)cfg.d);
        cudaFree(cfg.r[0]);
        cudaFree(cfg.w[0]);
        cudaFree(cfg.split_acc);
        cudaFree(cfg.partial);
        cudaFree(d_cfg);
        cudaFree(d_st);
        cudaFreeHost(h_st);
    }
    int kind() const override { return kBatchPpr; }
    int lanes() const override { return kColLanes; }
    const BatchStatus* host() const override { return h_st; }
    size_t device_bytes() const override { return bytes; }
    size_t lane_bytes() const override { return (size_t)cfg.n * 16; }
    int kernels_per_iter() const override { return 5; }

    int init(gbk_matrix a, const BatchOptions& o, cudaStream_t s) {
        A = a;
        opt = o;
        int rc = init_col_cfg(A, o, true, cfg, items, s);
        if (rc) return rc;
        rc = ensure_csc(A, s);  // column degrees
        if (rc) return rc;
        const int64_t n = cfg.n;
        const size_t nn = (size_t)std::max<int64_t>(n, 1);
        int32_t* cdeg = nullptr;
        float* d = nullptr;
        GBK_CUDA(cudaMalloc(&cdeg, 4 * nn));
        GBK_CUDA(cudaMalloc(&d, 4 * nn));
        cfg.cdeg = cdeg;
        cfg.d = d;
        if (n > 0) {
            k_ppr_degree<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A->csc.ptr, n, o.damping, cdeg, d);
            GBK_LAUNCHED();
        }
        GBK_CUDA(cudaMalloc(&cfg.r[0], 2 * 4 * 32 * nn));
        cfg.r[1] = cfg.r[0] + 32 * nn;
        GBK_CUDA(cudaMalloc(&cfg.w[0], 2 * 4 * 32 * nn));
        cfg.w[1] = cfg.w[0] + 32 * nn;
        GBK_CUDA(cudaMemsetAsync(cfg.r[0], 0, 2 * 4 * 32 * nn, s));
        GBK_CUDA(cudaMemsetAsync(cfg.w[0], 0, 2 * 4 * 32 * nn, s));
        GBK_CUDA(cudaMalloc(&cfg.split_acc, 4 * 32 * (size_t)std::max<int64_t>(items.nslots, 1)));
        grid_main = persistent_blocks((const void*)k_ppr_spmm, kBT);
        grid_fix = (int)std::max<int64_t>(1, std::min<int64_t>(grid_main, (items.nsplit * 32 + kBT - 1) / kBT));
        grid_upd = persistent_blocks((const void*)k_ppr_update, kBT);
        cfg.parts_main = grid_upd;
        GBK_CUDA(cudaMalloc(&cfg.partial, sizeof(double) * 64 * grid_upd));
        GBK_CUDA(cudaMalloc(&d_cfg, sizeof(ColCfg)));
        GBK_CUDA(cudaMalloc(&d_st, sizeof(PprState)));
        GBK_CUDA(cudaMallocHost(&h_st, sizeof(BatchStatus)));
        memset(h_st, 0, sizeof(BatchStatus));
        GBK_CUDA(cudaMemcpyAsync(d_cfg, &cfg, sizeof(ColCfg), cudaMemcpyHostToDevice, s));
        PprState init{};
        init.damping = o.damping;
        init.tol = o.tol;
        init.itermax = o.itermax;
        init.launch_budget = 1;
        for (int k = 0; k < 32; ++k) init.result_buf[k] = -1;
        GBK_CUDA(cudaMemcpyAsync(d_st, &init, sizeof(PprState), cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        bytes = 8 * nn + 4 * 4 * 32 * nn + 4 * 32 * (size_t)items.nslots + 20 * (size_t)items.nitems;
        return build_loop(loop, [this](cudaStream_t cs, cudaGraphConditionalHandle h) -> int {
            k_ppr_spmm<<<grid_main, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_ppr_fix<<<grid_fix, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_ppr_update<<<grid_upd, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_ppr_control<<<1, 1024, 0, cs>>>(d_cfg, d_st, h);
            GBK_LAUNCH_CHECK();
            return GBK_SUCCESS;
        });
    }

    int admit(unsigned long long mask, const int32_t* src, cudaStream_t s) override {
        mask &= 0xffffffffull;
        if (!mask) return GBK_SUCCESS;
        Lanes32 l{};
        for (int k = 0; k < kColLanes; ++k)
            if ((mask >> k) & 1) {
                GBK_REQUIRE(src[k] >= 0 && src[k] < cfg.n, GBK_INVALID_INDEX,
                            "batched PPR: seed %d out of range [0, %lld)", src[k], (long long)cfg.n);
                l.v[k] = src[k];
            }
        Lanes32 nlist{};
        int nl = 0;
        for (int k = 0; k < kColLanes; ++k)
            if ((mask >> k) & 1) nlist.v[nl++] = k;
        const int64_t total = cfg.n * nl;
        const unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)num_sms() * 16);
        if (g > 0) {
            k_ppr_init_cols<<<g, 256, 0, s>>>(d_cfg, d_st, nlist, nl, l);
            GBK_LAUNCHED();
        }
        k_ppr_admit<<<1, 32, 0, s>>>(d_cfg, d_st, (unsigned)mask, l, (double)opt.damping, opt.tol, opt.itermax);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }

    int launch(int budget, bool stop_on_finish, cudaStream_t s) override {
        k_set_launch<PprState><<<1, 1, 0, s>>>(d_st, budget, stop_on_finish ? 1 : 0);
        GBK_LAUNCHED();
        return run_loop(loop, &d_st->st, h_st, budget, stop_on_finish, s);
    }

    int extract(int lane_lo, int nl, void* dst, int64_t stride, cudaStream_t s) override {
        GBK_REQUIRE(lane_lo >= 0 && nl >= 0 && lane_lo + nl <= kColLanes, GBK_INVALID_INDEX,
                    "PPR extract: bad lanes");
        if (nl == 0 || cfg.n == 0) return GBK_SUCCESS;
        k_extract_cols<float><<<(unsigned)((cfg.n + 31) / 32), dim3(32, 8), 0, s>>>(
            cfg.r[0], cfg.r[1], d_st->result_buf, cfg.n, lane_lo, nl, (float*)dst, stride);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }

    int digest(unsigned long long mask, LaneDigest* d_out, cudaStream_t s) override {
        return launch_digest<1>(cfg.r[0], cfg.r[1], d_st->result_buf, cfg.n, 0, mask & 0xffffffffull, kColLanes,
                                d_out, s);
    }

    int release(unsigned long long mask, cudaStream_t s) override {
        k_cols_release<<<1, 1, 0, s>>>(&d_st->st, mask);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }
};

// ----------------------------------------------------------------------------
// 32-column SSSP (label-correcting push, int32 distances)

struct SsspState {
    BatchStatus st;
    int32_t src[32];
    unsigned alive;
    int32_t launch_budget, stop_on_finish, max_iter;
};

__device__ __forceinline__ int32_t weight_at(const ColCfg* __restrict__ cfg, int64_t e) {
    return cfg->vtype == GBK_F32 ? (int32_t)__ldcs((const float*)cfg->val + e) : __ldcs((const int32_t*)cfg->val + e);
}

// One warp per work item of a row whose distance changed in some lane:
// lane k relaxes the row's edges for column k and the warp ORs the lanes
// that improved into the neighbour's next change mask.
__global__ void __launch_bounds__(kBT) k_sssp_push(const ColCfg* __restrict__ cfg, const SsspState* __restrict__ st) {
    const unsigned act = (unsigned)st->st.active;
    if (!act) return;
    const int lane = threadIdx.x & 31;
    const int cur = st->st.iter & 1;
    const uint32_t* __restrict__ chg_in = cfg->chg[cur];
    uint32_t* chg_out = cfg->chg[cur ^ 1];
    int32_t* dist = cfg->dist;
    const int32_t* __restrict__ rp = cfg->rp;
    const int32_t* __restrict__ col = cfg->col;
    const int C = cfg->item_edges;
    const int64_t gw = ((int64_t)blockIdx.x * kBT + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kBT) >> 5;
    for (int64_t it = gw; it < cfg->nitems; it += nw) {
        const int32_t row = cfg->item_row[it];
        const uint32_t cm = chg_in[row] & act;
        if (!cm) continue;
        const bool mine = (cm >> lane) & 1;
        const int32_t dv = mine ? *((volatile const int32_t*)dist + (int64_t)row * 32 + lane) : INT_MAX;
        const int32_t beg = cfg->item_beg[it];
        const int32_t end = min(beg + C, rp[row + 1]);
        for (int32_t e0 = beg; e0 < end; e0 += 32) {
            const int cnt = min(32, end - e0);
            int32_t cl = 0, wl = 0;
            if (lane < cnt) {
                cl = __ldcs(col + e0 + lane);
                wl = weight_at(cfg, e0 + lane);
            }
            for (int j = 0; j < cnt; ++j) {
                const int32_t u = __shfl_sync(kFull, cl, j);
                const int32_t wt = __shfl_sync(kFull, wl, j);
                bool imp = false;
                if (mine) {
                    const int32_t cand = elem_add(dv, wt);
                    int32_t* p = dist + (int64_t)u * 32 + lane;
                    if (cand < *((volatile int32_t*)p)) imp = atomicMin(p, cand) > cand;
                }
                const unsigned m = __ballot_sync(kFull, imp);
                if (m && lane == 0) atomicOr(chg_out + u, m);
            }
        }
    }
}

__global__ void __launch_bounds__(kBT) k_sssp_finalize(const ColCfg* __restrict__ cfg, SsspState* st) {
    __shared__ unsigned s_alive;
    if (threadIdx.x == 0) s_alive = 0;
    __syncthreads();
    const int cur = st->st.iter & 1;
    uint32_t* chg_in = cfg->chg[cur];
    const uint32_t* __restrict__ chg_out = cfg->chg[cur ^ 1];
    unsigned alive = 0;
    if (st->st.active) {
        for (int64_t v = (int64_t)blockIdx.x * kBT + threadIdx.x; v < cfg->n; v += (int64_t)gridDim.x * kBT) {
            alive |= chg_out[v];
            if (chg_in[v]) chg_in[v] = 0;
        }
    }
    alive = __reduce_or_sync(kFull, alive);
    if ((threadIdx.x & 31) == 0 && alive) atomicOr(&s_alive, alive);
    __syncthreads();
    if (threadIdx.x == 0 && s_alive) atomicOr(&st->alive, s_alive);
}

__global__ void k_sssp_control(SsspState* st, cudaGraphConditionalHandle h) {
    const int k = threadIdx.x;  // 32 threads
    const unsigned act = (unsigned)st->st.active, alive = st->alive;
    unsigned fin = 0;
    if ((act >> k) & 1) {
        st->st.iters[k] += 1;
        if (!((alive >> k) & 1) || st->st.iters[k] >= st->max_iter) fin = 1u << k;
    }
    fin = __reduce_or_sync(kFull, fin);
    if (k == 0) {
        st->st.active = act & ~fin;
        st->st.finished |= fin;
        st->st.iter += 1;
        st->st.launch_iters += 1;
        st->alive = 0;
        const bool cont = st->st.active != 0 && st->st.launch_iters < st->launch_budget &&
                          !(st->stop_on_finish && fin);
        if (h) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

__global__ void k_sssp_init_cols(const ColCfg* __restrict__ cfg, Lanes32 lanes, int nl, Lanes32 src) {
    const int64_t total = cfg->n * nl;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i / nl;
        const int k = lanes.v[i - v * nl];
        cfg->dist[v * 32 + k] = (v == src.v[k]) ? 0 : INT_MAX;
    }
}

__global__ void k_sssp_admit(const ColCfg* __restrict__ cfg, SsspState* st, unsigned mask, Lanes32 src, int max_iter) {
    const int k = threadIdx.x;
    if (k == 0) st->max_iter = max_iter;
    if ((mask >> k) & 1) {
        st->src[k] = src.v[k];
        st->st.iters[k] = 0;
        atomicOr(cfg->chg[st->st.iter & 1] + src.v[k], 1u << k);
    }
    __syncwarp();
    if (k == 0) {
        st->st.active |= mask;
        st->st.finished &= ~(unsigned long long)mask;
    }
}

struct SsspBatch final : Batch {
    gbk_matrix A = nullptr;
    BatchOptions opt;
    ColCfg cfg{};
    RowItems items;
    ColCfg* d_cfg = nullptr;
    SsspState* d_st = nullptr;
    BatchStatus* h_st = nullptr;
    LoopGraph loop;
    int grid_main = 0, grid_fin = 0;
    size_t bytes = 0;

    ~SsspBatch() override {
        items.release();
        cudaFree(cfg.dist);
        cudaFree(cfg.chg[0]);
        cudaFree(d_cfg);
        cudaFree(d_st);
        cudaFreeHost(h_st);
    }
    int kind() const override { return kBatchSssp; }
    int lanes() const override { return kColLanes; }
    const BatchStatus* host() const override { return h_st; }
    size_t device_bytes() const override { return bytes; }
    size_t lane_bytes() const override { return (size_t)cfg.n * 4; }
    int kernels_per_iter() const override { return 3; }

    int max_iter() const {
        return opt.sssp_max_iter > 0 ? opt.sssp_max_iter
                                     : (int)std::min<int64_t>(std::max<int64_t>(cfg.n, 1), INT_MAX);
    }

    int init(gbk_matrix a, const BatchOptions& o, cudaStream_t s) {
        A = a;
        opt = o;
        int rc = init_col_cfg(A, o, false, cfg, items, s);
        if (rc) return rc;
        const size_t nn = (size_t)std::max<int64_t>(cfg.n, 1);
        GBK_CUDA(cudaMalloc(&cfg.dist, 4 * 32 * nn));
        GBK_CUDA(cudaMalloc(&cfg.chg[0], 2 * 4 * nn));
        cfg.chg[1] = cfg.chg[0] + nn;
        GBK_CUDA(cudaMemsetAsync(cfg.chg[0], 0, 2 * 4 * nn, s));
        grid_main = persistent_blocks((const void*)k_sssp_push, kBT);
        grid_fin = persistent_blocks((const void*)k_sssp_finalize, kBT);
        GBK_CUDA(cudaMalloc(&d_cfg, sizeof(ColCfg)));
        GBK_CUDA(cudaMalloc(&d_st, sizeof(SsspState)));
        GBK_CUDA(cudaMallocHost(&h_st, sizeof(BatchStatus)));
        memset(h_st, 0, sizeof(BatchStatus));
        GBK_CUDA(cudaMemcpyAsync(d_cfg, &cfg, sizeof(ColCfg), cudaMemcpyHostToDevice, s));
        SsspState init{};
        init.launch_budget = 1;
        init.max_iter = max_iter();
        GBK_CUDA(cudaMemcpyAsync(d_st, &init, sizeof(SsspState), cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        bytes = 4 * 32 * nn + 8 * nn + 20 * (size_t)items.nitems;
        return build_loop(loop, [this](cudaStream_t cs, cudaGraphConditionalHandle h) -> int {
            k_sssp_push<<<grid_main, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_sssp_finalize<<<grid_fin, kBT, 0, cs>>>(d_cfg, d_st);
            GBK_LAUNCH_CHECK();
            k_sssp_control<<<1, 32, 0, cs>>>(d_st, h);
            GBK_LAUNCH_CHECK();
            return GBK_SUCCESS;
        });
    }

    int admit(unsigned long long mask, const int32_t* src, cudaStream_t s) override {
        mask &= 0xffffffffull;
        if (!mask) return GBK_SUCCESS;
        Lanes32 l{};
        for (int k = 0; k < kColLanes; ++k)
            if ((mask >> k) & 1) {
                GBK_REQUIRE(src[k] >= 0 && src[k] < cfg.n, GBK_INVALID_INDEX,
                            "batched SSSP: source %d out of range [0, %lld)", src[k], (long long)cfg.n);
                l.v[k] = src[k];
            }
        Lanes32 nlist{};
        int nl = 0;
        for (int k = 0; k < kColLanes; ++k)
            if ((mask >> k) & 1) nlist.v[nl++] = k;
        const int64_t total = cfg.n * nl;
        const unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)num_sms() * 16);
        if (g > 0) {
            k_sssp_init_cols<<<g, 256, 0, s>>>(d_cfg, nlist, nl, l);
            GBK_LAUNCHED();
        }
        k_sssp_admit<<<1, 32, 0, s>>>(d_cfg, d_st, (unsigned)mask, l, max_iter());
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }

    int launch(int budget, bool stop_on_finish, cudaStream_t s) override {
        k_set_launch<SsspState><<<1, 1, 0, s>>>(d_st, budget, stop_on_finish ? 1 : 0);
        GBK_LAUNCHED();
        return run_loop(loop, &d_st->st, h_st, budget, stop_on_finish, s);
    }

    int extract(int lane_lo, int nl, void* dst, int64_t stride, cudaStream_t s) override {
        GBK_REQUIRE(lane_lo >= 0 && nl >= 0 && lane_lo + nl <= kColLanes, GBK_INVALID_INDEX,
                    "SSSP extract: bad lanes");
        if (nl == 0 || cfg.n == 0) return GBK_SUCCESS;
        k_extract_cols<int32_t><<<(unsigned)((cfg.n + 31) / 32), dim3(32, 8), 0, s>>>(
            cfg.dist, cfg.dist, nullptr, cfg.n, lane_lo, nl, (int32_t*)dst, stride);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }

    int digest(unsigned long long mask, LaneDigest* d_out, cudaStream_t s) override {
        return launch_digest<2>(cfg.dist, nullptr, nullptr, cfg.n, 0, mask & 0xffffffffull, kColLanes, d_out, s);
    }

    int release(unsigned long long mask, cudaStream_t s) override {
        k_cols_release<<<1, 1, 0, s>>>(&d_st->st, mask);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }
};

template <typename B>
int make_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s) {
    GBK_REQUIRE(A && out, GBK_NULL_POINTER, "batched traversal: NULL argument");
    B* b = new B();
    const int rc = b->init(A, o, s);
    if (rc) {
        delete b;
        return rc;
    }
    *out = b;
    return GBK_SUCCESS;
}

// One-shot driver: admit lanes 0..k-1, run the graph until every lane ends,
// copy the results out, release the lanes.
int run_one_shot(Batch* b, int k, const int32_t* src, void* out, int64_t stride, int32_t* iters, bool extract,
                 cudaStream_t s) {
    std::vector<int32_t> lane_src(b->lanes(), 0);
    for (int i = 0; i < k; ++i) lane_src[i] = src[i];
    const unsigned long long mask = k >= 64 ? ~0ull : ((1ull << k) - 1);
    int rc = b->admit(mask, lane_src.data(), s);
    if (rc) return rc;
    GBK_CUDA(cudaStreamSynchronize(s));
    const int it0 = b->host()->iter;
    rc = b->launch(INT_MAX, false, s);
    if (rc) return rc;
    GBK_CUDA(cudaStreamSynchronize(s));
    const BatchStatus* st = b->host();
    count_launch(b->kernels_per_iter() * (st->iter - it0));
    GBK_REQUIRE((st->active & mask) == 0, GBK_PANIC, "batched traversal: lanes still active after the loop");
    if (extract) {
        rc = b->extract(0, k, out, stride, s);
        if (rc) return rc;
    }
    if (iters)
        for (int i = 0; i < k; ++i) iters[i] = st->iters[i];
    rc = b->release(mask, s);
    if (rc) return rc;
    GBK_CUDA(cudaStreamSynchronize(s));
    return GBK_SUCCESS;
}

}  // namespace

int make_bfs_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s) {
    return make_batch<BfsBatch>(A, o, out, s);
}
int make_ppr_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s) {
    return make_batch<PprBatch>(A, o, out, s);
}
int make_sssp_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s) {
    return make_batch<SsspBatch>(A, o, out, s);
}
int bfs_batch_set_levels(Batch* b, int32_t* levels, int64_t stride, cudaStream_t s) {
    GBK_REQUIRE(b && b->kind() == kBatchBfs, GBK_INVALID_OBJECT, "not a BFS batch");
    return static_cast<BfsBatch*>(b)->set_levels(levels, stride, s);
}

BatchOptions base_options(gbk_matrix A, int kind) {
    return A->batch_tuned[kind] ? A->batch_tuned_opt[kind] : BatchOptions{};
}

void free_batches(gbk_matrix A) {
    for (auto& p : A->batch) {
        delete p;
        p = nullptr;
    }
}

}  // namespace gbk

using namespace gbk;

namespace {

// The matrix keeps one batch per kind for the one-shot calls; it is rebuilt
// when the options it was made with change.
int cached_batch(gbk_matrix A, int kind, const BatchOptions& o, Batch** out, cudaStream_t s) {
    Batch*& slot = A->batch[kind];
    BatchOptions& have = A->batch_opt[kind];
    const bool same = slot && have.item_edges == o.item_edges && have.damping == o.damping && have.tol == o.tol &&
                      have.itermax == o.itermax && have.sssp_max_iter == o.sssp_max_iter;
    if (!same) {
        delete slot;
        slot = nullptr;
        const int rc = kind == kBatchBfs   ? make_bfs_batch(A, o, &slot, s)
                       : kind == kBatchPpr ? make_ppr_batch(A, o, &slot, s)
                                           : make_sssp_batch(A, o, &slot, s);
        if (rc) return rc;
        have = o;
    }
    *out = slot;
    return GBK_SUCCESS;
}

}  // namespace

extern "C" {

int gbk_msbfs(gbk_matrix A, const int32_t* sources, int nsources, int32_t* levels, int direction, int32_t* depths,
              void* stream) {
    GBK_REQUIRE(A && (nsources == 0 || (sources && levels)), GBK_NULL_POINTER, "gbk_msbfs: NULL argument");
    GBK_REQUIRE(nsources >= 0 && nsources <= kBfsLanes, GBK_INVALID_VALUE, "gbk_msbfs: nsources must be in [0, 64]");
    GBK_REQUIRE(direction >= 0 && direction <= 2, GBK_INVALID_VALUE, "gbk_msbfs: direction must be 0, 1 or 2");
    GBK_REQUIRE(A->csr.nrows == A->csr.ncols, GBK_DIMENSION_MISMATCH, "gbk_msbfs: matrix must be square");
    if (nsources == 0) return GBK_SUCCESS;
    for (int i = 0; i < nsources; ++i)
        GBK_REQUIRE(sources[i] >= 0 && sources[i] < A->csr.nrows, GBK_INVALID_INDEX,
                    "gbk_msbfs: source %d out of range", sources[i]);
    cudaStream_t s = (cudaStream_t)stream;
    const BatchOptions o = base_options(A, kBatchBfs);
    Batch* b = nullptr;
    int rc = cached_batch(A, kBatchBfs, o, &b, s);
    if (rc) return rc;
    BfsBatch* bb = static_cast<BfsBatch*>(b);
    rc = bb->set_mode(direction == 0 ? o.bfs_direction : direction, o.bfs_alpha, o.bfs_beta, s);
    if (rc) return rc;
    rc = bb->set_levels(levels, A->csr.nrows, s);
    if (rc) return rc;
    rc = run_one_shot(b, nsources, sources, nullptr, 0, depths, false, s);
    const int rc2 = bb->set_levels(nullptr, 0, s);
    return rc ? rc : rc2;
}

int gbk_ppr(gbk_matrix A, const int32_t* seeds, int nseeds, double damping, double tol, int itermax, float* ranks,
            int32_t* iters, void* stream) {
    GBK_REQUIRE(A && (nseeds == 0 || (seeds && ranks)), GBK_NULL_POINTER, "gbk_ppr: NULL argument");
    GBK_REQUIRE(nseeds >= 0 && nseeds <= kColLanes, GBK_INVALID_VALUE, "gbk_ppr: nseeds must be in [0, 32]");
    GBK_REQUIRE(damping > 0 && damping < 1 && itermax >= 1, GBK_INVALID_VALUE,
                "gbk_ppr: damping must be in (0, 1) and itermax >= 1");
    if (nseeds == 0) return GBK_SUCCESS;
    for (int i = 0; i < nseeds; ++i)
        GBK_REQUIRE(seeds[i] >= 0 && seeds[i] < A->csr.nrows, GBK_INVALID_INDEX, "gbk_ppr: seed %d out of range",
                    seeds[i]);
    cudaStream_t s = (cudaStream_t)stream;
    BatchOptions o = base_options(A, kBatchPpr);
    o.damping = (float)damping;
    o.tol = tol;
    o.itermax = itermax;
    Batch* b = nullptr;
    int rc = cached_batch(A, kBatchPpr, o, &b, s);
    if (rc) return rc;
    return run_one_shot(b, nseeds, seeds, ranks, A->csr.nrows, iters, true, s);
}

int gbk_sssp_multi(gbk_matrix A, const int32_t* sources, int nsources, int32_t* dist, int32_t* iters, void* stream) {
    GBK_REQUIRE(A && (nsources == 0 || (sources && dist)), GBK_NULL_POINTER, "gbk_sssp_multi: NULL argument");
    GBK_REQUIRE(nsources >= 0 && nsources <= kColLanes, GBK_INVALID_VALUE,
                "gbk_sssp_multi: nsources must be in [0, 32]");
    if (nsources == 0) return GBK_SUCCESS;
    for (int i = 0; i < nsources; ++i)
        GBK_REQUIRE(sources[i] >= 0 && sources[i] < A->csr.nrows, GBK_INVALID_INDEX,
                    "gbk_sssp_multi: source %d out of range", sources[i]);
    cudaStream_t s = (cudaStream_t)stream;
    const BatchOptions o = base_options(A, kBatchSssp);
    Batch* b = nullptr;
    int rc = cached_batch(A, kBatchSssp, o, &b, s);
    if (rc) return rc;
    return run_one_shot(b, nsources, sources, dist, A->csr.nrows, iters, true, s);
}

}  // extern "C"

namespace {

// Device time of one one-shot run (events on s around a synchronising call).
int time_one_shot(Batch* b, int k, const int32_t* src, void* out, int64_t stride, bool extract, cudaStream_t s,
                  float* ms) {
    cudaEvent_t e0, e1;
    GBK_CUDA(cudaEventCreate(&e0));
    GBK_CUDA(cudaEventCreate(&e1));
    int rc = run_one_shot(b, k, src, out, stride, nullptr, extract, s);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 2 && !rc; ++r) {
        cudaEventRecord(e0, s);
        rc = run_one_shot(b, k, src, out, stride, nullptr, extract, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        best = std::min(best, t);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = best;
    return rc;
}

}  // namespace

extern "C" int gbk_batch_autotune(gbk_matrix A, int kind, const int32_t* sources, int nsources,
                                  gbk_batch_tune_result* out, void* stream) {
    GBK_REQUIRE(A && sources && out, GBK_NULL_POINTER, "gbk_batch_autotune: NULL argument");
    GBK_REQUIRE(kind >= 0 && kind <= 2, GBK_INVALID_VALUE, "gbk_batch_autotune: kind must be 0, 1 or 2");
    const int lanes = kind == kBatchBfs ? kBfsLanes : kColLanes;
    GBK_REQUIRE(nsources >= 1 && nsources <= lanes, GBK_INVALID_VALUE, "gbk_batch_autotune: 1 to %d sources", lanes);
    const int64_t n = A->csr.nrows;
    for (int i = 0; i < nsources; ++i)
        GBK_REQUIRE(sources[i] >= 0 && sources[i] < n, GBK_INVALID_INDEX, "gbk_batch_autotune: source out of range");
    cudaStream_t s = (cudaStream_t)stream;
    memset(out, 0, sizeof(*out));
    out->kind = kind;
    void* buf = nullptr;
    GBK_CUDA(cudaMalloc(&buf, 4 * (size_t)std::max<int64_t>(n, 1) * nsources));
    BatchOptions best = base_options(A, kind);
    float best_ms = 1e30f;
    int rc = GBK_SUCCESS;
    if (kind == kBatchBfs) {
        const int dirs[6] = {0, 0, 0, 0, 1, 2};
        const int alphas[6] = {2, 4, 8, 14, 4, 4};
        Batch* b = nullptr;
        rc = cached_batch(A, kBatchBfs, base_options(A, kBatchBfs), &b, s);
        BfsBatch* bb = static_cast<BfsBatch*>(b);
        if (!rc) rc = bb->set_levels((int32_t*)buf, n, s);
        for (int c = 0; c < 6 && !rc; ++c) {
            rc = bb->set_mode(dirs[c], alphas[c], best.bfs_beta, s);
            float ms = 0;
            if (!rc) rc = time_one_shot(b, nsources, sources, nullptr, 0, false, s, &ms);
            out->candidate_ms[c] = ms;
            if (!rc && ms < best_ms) {
                best_ms = ms;
                best.bfs_direction = dirs[c];
                best.bfs_alpha = alphas[c];
            }
        }
        if (b) {
            const int rc2 = bb->set_levels(nullptr, 0, s);
            if (!rc) rc = rc2;
        }
        out->ncandidates = 6;
    } else {
        const int sizes[5] = {64, 128, 256, 512, 1024};
        for (int c = 0; c < 5 && !rc; ++c) {
            BatchOptions o = base_options(A, kind);
            o.item_edges = sizes[c];
            Batch* b = nullptr;
            rc = kind == kBatchPpr ? make_ppr_batch(A, o, &b, s) : make_sssp_batch(A, o, &b, s);
            float ms = 0;
            if (!rc) rc = time_one_shot(b, nsources, sources, buf, n, true, s, &ms);
            delete b;
            out->candidate_ms[c] = ms;
            if (!rc && ms < best_ms) {
                best_ms = ms;
                best.item_edges = sizes[c];
            }
        }
        out->ncandidates = 5;
    }
    cudaFree(buf);
    if (rc) return rc;
    A->batch_tuned[kind] = true;
    A->batch_tuned_opt[kind] = best;
    out->item_edges = best.item_edges;
    out->bfs_direction = best.bfs_direction;
    out->bfs_alpha = best.bfs_alpha;
    out->best_ms = best_ms;
    return GBK_SUCCESS;
}
