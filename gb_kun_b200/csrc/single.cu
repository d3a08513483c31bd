// Single-query traversals with the whole iteration loop on the device.
//
// The reference runs its algorithms as one GraphBLAS call per step with a
// host read of the convergence scalar every iteration (bfs_blast,
// algorithms/bfs/bfs.hpp:94-142; sssp_bellman_ford_blast,
// algorithms/sssp/sssp_blast.hpp:8-72; cc, algorithms/cc/cc.hpp:12-119); the
// drop-in header runs exactly that sequence.  These entry points compute the
// same outputs with fused device loops:
//
//  * gbk_bfs_levels: direction-optimising BFS along CSR rows (the vxm of
//    bfs_blast), levels 1 for the source, k + 1 at distance k, 0 unreached.
//    Each level expands the frontier top-down from a queue of its vertices
//    or bottom-up over the unvisited vertices' in-edges (CSC) testing a
//    frontier bitmap, and records every vertex it reaches in both the next
//    queue and the next bitmap, so switching direction needs no conversion.
//    A one-warp control kernel switches on the frontier's out-edges against
//    the unvisited vertices' out-edges (Beamer's rule) and ends the loop;
//    the level's kernels form the body of one CUDA graph whose `while` node
//    the control kernel drives, so a whole BFS is one graph launch.
//  * gbk_sssp_dist: the distances of sssp_bellman_ford_blast by a
//    label-correcting near-far worklist: each round relaxes the out-edges
//    of the near vertices whose distance dropped (an atomic min per edge,
//    bitmaps so each improved vertex is queued once), one graph launch for
//    all rounds.
//  * gbk_pagerank: page_rank_sinks (algorithms/pr/pr.hpp:20-153): each
//    iteration is the matrix's SpMV (plus-second, its autotuned format), one
//    element-wise pass (teleport, |r_old - r_new|, the next r ./ d and the
//    sink sum, per-block partials) and a one-block control kernel summing
//    the partials in a fixed order; the iterations after the first run as
//    one CUDA graph.
//  * gbk_cc_labels: connected components as min-vertex-id labels (the fixed
//    point FastSV reaches on an undirected graph) by lock-free union-find
//    with sampled linking (Sutton, Ben-Nun and Barak, "Optimizing Parallel
//    Graph Connectivity Computation via Subgraph Sampling", IPDPS 2018):
//    every vertex first links along its first two entries, the largest
//    component is found from a sample of 1024 vertices, and only vertices
//    outside it link along their remaining entries (on a symmetric pattern
//    the other end of every skipped edge links it).  Links always put the
//    larger of two roots under the smaller one (compare-and-swap), so a
//    component's root is its smallest vertex and the labels do not depend
//    on the order of the links.  A non-symmetric pattern links every entry
//    in both directions, which gives its weakly connected components.
//
// Frontier expansion is load-balanced the same way for BFS and SSSP: a warp
// takes 32 frontier vertices; rows under kHeavy entries are spread over the
// warp's lanes edge by edge (a warp scan of their lengths and a 5-step
// search for each lane's row), longer rows are cut into kChunk-entry chunks
// that a second kernel of the same level hands out one per warp.
#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

constexpr int kT = 256;
constexpr unsigned kAll = 0xffffffffu;
constexpr int kHeavy = 32;   // rows with at least this many entries are cut into chunks
constexpr int kChunk = 256;  // entries per chunk

int blocks_for_sm(const void* kern) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kT, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * num_sms();
}

unsigned grid1(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kT - 1) / kT); }

// A graph whose root is a `while` node around the kernels `body` launches on
// the stream it is given (captured once; the last of them sets the
// condition from the device).
template <typename Body>
int build_loop_graph(cudaGraph_t* graph, cudaGraphExec_t* exec, Body body) {
    GBK_CUDA(cudaGraphCreate(graph, 0));
    cudaGraphConditionalHandle handle;
    GBK_CUDA(cudaGraphConditionalHandleCreate(&handle, *graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    GBK_CUDA(cudaGraphAddNode(&node, *graph, nullptr, 0, &p));
    cudaGraph_t bodyg = p.conditional.phGraph_out[0];
    cudaStream_t cs;
    GBK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return cuda_fail(e, "cudaStreamBeginCaptureToGraph", __FILE__, __LINE__);
    }
    body(cs, handle);
    cudaError_t le = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    if (le != cudaSuccess) return cuda_fail(le, "loop body launch", __FILE__, __LINE__);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    GBK_CUDA(cudaGraphInstantiate(exec, *graph, 0));
    return GBK_SUCCESS;
}

bool host_loop_mode() {
    const char* e1 = getenv("GBK_HOST_LOOP");
    const char* e2 = getenv("GBK_BATCH_HOST_LOOP");
    return (e1 && e1[0] == '1') || (e2 && e2[0] == '1');
}

}  // namespace

// One loop kept per matrix: its scratch (allocated once) and its
// instantiated graph, whose kernel arguments point into that scratch, so a
// call only launches the init kernel and the graph (building and
// instantiating the graph took as long as a whole BFS at R-MAT scale 23).
struct CachedLoop {
    void* mem = nullptr;
    size_t bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t key = -1;  // what the graph was built for (PageRank: the matrix's format generation)
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        key = -1;
    }
    void release() {
        drop_graph();
        cudaFree(mem);
        mem = nullptr;
        bytes = 0;
    }
};

struct SingleCache {
    CachedLoop bfs, sssp, pr;
    double mean_weight = -1.0;  // sampled mean edge value (SSSP's automatic delta)
};

void free_single_cache(gbk_matrix A) {
    if (!A->single) return;
    A->single->bfs.release();
    A->single->sssp.release();
    A->single->pr.release();
    delete A->single;
    A->single = nullptr;
}

namespace {

SingleCache& single_cache(gbk_matrix A) {
    if (!A->single) A->single = new SingleCache();
    return *A->single;
}

// The loop's scratch: allocated on first use (or grown), then kept.
int loop_scratch(CachedLoop& L, size_t bytes) {
    if (L.mem && L.bytes >= bytes) return GBK_SUCCESS;
    L.release();
    GBK_CUDA(cudaMalloc(&L.mem, bytes));
    L.bytes = bytes;
    return GBK_SUCCESS;
}

// Runs the loop on s: the cached graph (built on first use, or again when
// `key` changed), or the host loop for profilers.
template <typename Body>
int launch_loop(CachedLoop& L, int64_t key, cudaStream_t s, const int32_t* d_cont, Body body) {
    if (host_loop_mode()) {
        for (;;) {
            body(s, (cudaGraphConditionalHandle)0);
            GBK_CUDA(cudaGetLastError());
            int32_t cont = 0;
            GBK_CUDA(cudaMemcpyAsync(&cont, d_cont, 4, cudaMemcpyDeviceToHost, s));
            GBK_CUDA(cudaStreamSynchronize(s));
            if (!cont) return GBK_SUCCESS;
        }
    }
    if (L.exec && L.key != key) L.drop_graph();
    if (!L.exec) {
        const int rc = build_loop_graph(&L.graph, &L.exec, body);
        if (rc != GBK_SUCCESS) {
            L.drop_graph();
            return rc;
        }
        L.key = key;
    }
    GBK_CUDA(cudaGraphLaunch(L.exec, s));
    count_launch(1);
    return GBK_SUCCESS;
}

// ---- frontier expansion -----------------------------------------------------

struct Chunk {
    int32_t u;    // the row
    int32_t beg;  // its entries [beg, min(beg + kChunk, end of row))
};

__device__ __forceinline__ int32_t warp_incl_scan(int32_t x) {
    const int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(kAll, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Appends the lanes with `found` set to q (one atomic per warp).
__device__ __forceinline__ void queue_append(bool found, int32_t v, int32_t* q, int32_t* count) {
    const unsigned m = __ballot_sync(kAll, found);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    int32_t base = 0;
    if (lane == 0) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(kAll, base, 0);
    if (found) q[base + __popc(m & ((1u << lane) - 1u))] = v;
}

// The rows of the frontier qc[0, fc): rows under kHeavy entries edge by edge
// over the warp's lanes (op.edge(valid, value of the row, entry) on every
// lane), longer rows appended to `chunks` for expand_heavy.  Op::load(u)
// gives the per-row value passed to op.edge.
template <class Op>
__device__ void expand_light(const int32_t* __restrict__ qc, int32_t fc, const int32_t* __restrict__ rp,
                             Chunk* __restrict__ chunks, int32_t* nchunks, Op& op) {
    using V = typename Op::V;
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * kT + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * kT) >> 5;
    const int64_t ngroups = ((int64_t)fc + 31) / 32;
    for (int64_t c = gw; c < ngroups; c += nw) {
        const int64_t k = c * 32 + lane;
        const int32_t u = k < fc ? qc[k] : -1;
        const int32_t beg = u >= 0 ? rp[u] : 0, deg = u >= 0 ? rp[u + 1] - beg : 0;
        const bool heavy = deg >= kHeavy;
        const int32_t nch = heavy ? (deg + kChunk - 1) / kChunk : 0;
        const int32_t ich = warp_incl_scan(nch);
        const int32_t tch = __shfl_sync(kAll, ich, 31);
        if (tch) {
            int32_t base = 0;
            if (lane == 0) base = atomicAdd(nchunks, tch);
            base = __shfl_sync(kAll, base, 0);
            for (int32_t i = 0; i < nch; ++i) chunks[base + ich - nch + i] = Chunk{u, beg + i * kChunk};
        }
        const int32_t dl = heavy ? 0 : deg;
        const int32_t incl = warp_incl_scan(dl);
        const int32_t excl = incl - dl;
        const int32_t total = __shfl_sync(kAll, incl, 31);
        const V val = dl > 0 ? op.load(u) : V();
        for (int32_t t0 = 0; t0 < total; t0 += 32) {
            const int32_t t = t0 + lane;
            // the row of edge t: the first lane whose inclusive count exceeds t
            int j = 0;
            for (int s = 16; s; s >>= 1)
                if (__shfl_sync(kAll, incl, j + s - 1) <= t) j += s;
            j = min(j, 31);  // lanes past the end
            const int32_t eb = __shfl_sync(kAll, beg, j), ex = __shfl_sync(kAll, excl, j);
            const V vj = __shfl_sync(kAll, val, j);
            op.edge(t < total, vj, eb + (t - ex));
        }
    }
}

// The chunks expand_light appended, one warp per chunk.
template <class Op>
__device__ void expand_heavy(const Chunk* __restrict__ chunks, int32_t nch, const int32_t* __restrict__ rp, Op& op) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * kT + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * kT) >> 5;
    for (int64_t c = gw; c < nch; c += nw) {
        const Chunk ch = chunks[c];
        const int32_t end = min(ch.beg + kChunk, rp[ch.u + 1]);
        const typename Op::V val = op.load(ch.u);
        for (int32_t e0 = ch.beg; e0 < end; e0 += 32) op.edge(e0 + lane < end, val, e0 + lane);
    }
}

// Upper bound of the chunks one round appends: every row appears once per
// round and a row of d >= kHeavy entries gives ceil(d / kChunk) <= d / kHeavy.
int64_t max_chunks(int64_t nnz) { return nnz / kHeavy + 1; }

// ---- BFS --------------------------------------------------------------------

struct Bfs1State {
    int32_t level;        // level of the current frontier's vertices
    int32_t mode;         // 0 top-down (queue), 1 bottom-up (bitmap)
    int32_t fcount;       // vertices in the current frontier
    int32_t ncount;       // vertices reached this level (next frontier)
    long long nedges;     // out-edges of the next frontier
    long long uedges;     // out-edges of the vertices not reached yet
    int32_t cur;          // which queue is the current one
    int32_t bcur;         // which of the three bitmaps is the current one
    int32_t alpha, beta;  // top-down -> bottom-up when frontier edges > unvisited edges / alpha;
                          // back when frontier vertices < n / beta
    int32_t max_level;
    int32_t direction;    // 0 switch by the rule above, 1 top-down only, 2 bottom-up only
    int32_t nchunks;      // heavy-row chunks appended this level
    int32_t cont;         // another level runs
};

struct Bfs1Bufs {
    const int32_t* rp;   // CSR
    const int32_t* col;
    const int32_t* crp;  // CSC (in-edges)
    const int32_t* crow;
    int64_t n;
    int32_t* lv;
    int32_t* q[2];
    uint32_t* bm[3];
    int64_t nwords;
    Chunk* chunks;
};

// Per level: the queue and bitmap of the next frontier and the out-edges of
// the vertices recorded in them.
struct BfsNext {
    using V = int32_t;
    const int32_t* rp;
    const int32_t* col;
    int32_t* lv;
    int32_t next;  // the level being assigned
    int32_t* qn;
    uint32_t* bn;
    int32_t* ncount;
    long long edges;

    __device__ V load(int32_t) const { return 0; }
    __device__ __forceinline__ void record(bool found, int32_t v) {
        queue_append(found, v, qn, ncount);
        if (found) {
            atomicOr(bn + (v >> 5), 1u << (v & 31));
            edges += rp[v + 1] - rp[v];
        }
    }
    // top-down: claim an unvisited column
    __device__ __forceinline__ void edge(bool valid, V, int32_t e) {
        int32_t v = -1;
        bool found = false;
        if (valid) {
            v = col[e];
            found = lv[v] == 0 && atomicCAS(lv + v, 0, next) == 0;
        }
        record(found, v);
    }
    __device__ void flush(long long* total) {
        for (int o = 16; o; o >>= 1) edges += __shfl_xor_sync(kAll, edges, o);
        if ((threadIdx.x & 31) == 0 && edges) atomicAdd((unsigned long long*)total, (unsigned long long)edges);
    }
};

__device__ __forceinline__ BfsNext bfs_next(const Bfs1Bufs& b, Bfs1State* st) {
    return BfsNext{b.rp, b.col, b.lv, st->level + 1, b.q[st->cur ^ 1], b.bm[(st->bcur + 1) % 3], &st->ncount, 0};
}

// Top-down rows under kHeavy entries (and the chunks of longer ones), or the
// whole bottom-up level.
__global__ void __launch_bounds__(kT) k_bfs1_light(Bfs1Bufs b, Bfs1State* st) {
    BfsNext op = bfs_next(b, st);
    const uint32_t* bc = b.bm[st->bcur];
    uint32_t* bz = b.bm[(st->bcur + 2) % 3];  // the bitmap after next, cleared now
    const int64_t tid = (int64_t)blockIdx.x * kT + threadIdx.x, nth = (int64_t)gridDim.x * kT;
    for (int64_t i = tid; i < b.nwords; i += nth) bz[i] = 0;
    if (st->mode == 0) {
        expand_light(b.q[st->cur], st->fcount, b.rp, b.chunks, &st->nchunks, op);
    } else {
        // every unvisited vertex looks for an in-neighbour in the frontier:
        // rows under kHeavy entries by their lane, longer ones by the whole
        // warp 32 entries at a time
        const int lane = threadIdx.x & 31;
        const int64_t nr = (b.n + 31) / 32 * 32;
        for (int64_t v0 = tid; v0 < nr; v0 += nth) {
            const int32_t v = (int32_t)v0;
            const bool un = v0 < b.n && b.lv[v] == 0;
            const int32_t beg = un ? b.crp[v] : 0, deg = un ? b.crp[v + 1] - beg : 0;
            bool found = false;
            if (deg < kHeavy)
                for (int32_t e = beg; e < beg + deg; ++e) {
                    const int32_t u = b.crow[e];
                    if ((bc[u >> 5] >> (u & 31)) & 1u) {
                        found = true;
                        break;
                    }
                }
            unsigned hubs = __ballot_sync(kAll, deg >= kHeavy);
            while (hubs) {
                const int h = __ffs(hubs) - 1;
                hubs &= hubs - 1;
                const int32_t hb = __shfl_sync(kAll, beg, h), hd = __shfl_sync(kAll, deg, h);
                bool hf = false;
                for (int32_t e0 = 0; e0 < hd && !hf; e0 += 32) {
                    bool f = false;
                    if (e0 + lane < hd) {
                        const int32_t u = b.crow[hb + e0 + lane];
                        f = (bc[u >> 5] >> (u & 31)) & 1u;
                    }
                    hf = __any_sync(kAll, f);
                }
                if (lane == h) found = hf;
            }
            if (found) b.lv[v] = op.next;
            op.record(found, v);
        }
    }
    op.flush(&st->nedges);
}

__global__ void __launch_bounds__(kT) k_bfs1_heavy(Bfs1Bufs b, Bfs1State* st) {
    if (st->mode != 0) return;
    BfsNext op = bfs_next(b, st);
    expand_heavy(b.chunks, st->nchunks, b.rp, op);
    op.flush(&st->nedges);
}

__global__ void k_bfs1_control(Bfs1State* st, int64_t n, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    const int32_t nc = st->ncount;
    const long long ne = st->nedges;
    st->uedges -= ne;
    const bool cont = nc > 0 && st->level < st->max_level;
    if (cont && st->direction == 0) {
        if (st->mode == 0) {
            if (ne > st->uedges / st->alpha) st->mode = 1;
        } else if ((long long)nc * st->beta < n) {
            st->mode = 0;
        }
    }
    if (cont) {
        st->fcount = nc;
        st->level += 1;
        st->cur ^= 1;
        st->bcur = (st->bcur + 1) % 3;
    }
    st->ncount = 0;
    st->nedges = 0;
    st->nchunks = 0;
    st->cont = cont ? 1 : 0;
    if (h) cudaGraphSetConditional(h, cont ? 1u : 0u);
}

__global__ void k_bfs1_init(Bfs1Bufs b, Bfs1State* st, int32_t src, long long nnz, int alpha, int beta,
                            int direction) {
    const int64_t tid = (int64_t)blockIdx.x * kT + threadIdx.x, nth = (int64_t)gridDim.x * kT;
    for (int64_t i = tid; i < b.n; i += nth) b.lv[i] = i == src ? 1 : 0;
    for (int64_t i = tid; i < b.nwords; i += nth) {
        b.bm[0][i] = (i == (src >> 5)) ? (1u << (src & 31)) : 0u;
        b.bm[1][i] = 0;
        b.bm[2][i] = 0;
    }
    if (tid == 0) {
        b.q[0][0] = src;
        st->level = 1;
        st->direction = direction;
        st->mode = direction == 2 ? 1 : 0;
        st->fcount = 1;
        st->ncount = 0;
        st->nedges = 0;
        st->uedges = nnz - (b.rp[src + 1] - b.rp[src]);
        st->cur = 0;
        st->bcur = 0;
        st->alpha = alpha;
        st->beta = beta;
        st->max_level = b.n + 1 < (int64_t)INT32_MAX ? (int32_t)(b.n + 1) : INT32_MAX - 1;
        st->nchunks = 0;
    }
}

template <typename T>
__global__ void k_levels_out(const int32_t* __restrict__ lv, int64_t n, T* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
    if (i < n) out[i] = (T)lv[i];
}

// ---- SSSP -------------------------------------------------------------------
//
// Near-far worklist (Davidson, Baxter, Garland and Owens, "Work-Efficient
// Parallel GPU Methods for Single-Source Shortest Paths", IPDPS 2014): a
// vertex whose distance drops below the threshold joins the next round's
// (near) queue, one at or above it joins the far pile; when the near queue
// runs dry the threshold moves up by delta (or to the smallest far distance
// plus delta) and a split round moves the far vertices below it into the
// near queue.  Every improved vertex is expanded again later whatever its
// pile, so the fixpoint, and with it every distance, is the one plain
// Bellman-Ford reaches; the threshold only orders the work.

template <typename T>
struct Sssp1State {
    int32_t round;       // rounds run (expansions and splits)
    int32_t cur;         // which near queue is the current one
    int32_t fcount;      // vertices in the current near queue
    int32_t ncount;      // vertices appended to the next near queue
    int32_t max_rounds;
    int32_t nchunks;
    int32_t mode;        // 0 expand the near queue, 1 split the far pile
    int32_t fcur;        // which far buffer holds the pile
    int32_t farcount;    // vertices in the pile
    int32_t farnext;     // vertices kept by the running split
    int32_t use_far;     // 0: plain worklist (every improved vertex is near)
    T thr;               // near = distance below thr
    T thr_prev;          // the threshold before the running split
    T delta;
    T far_min;           // smallest distance kept in the pile by the running split
    int32_t cont;        // another round runs
};

template <typename T>
struct Sssp1Bufs {
    const int32_t* rp;
    const int32_t* col;
    const T* w;
    int64_t n;
    T* dist;
    int32_t* q[2];
    uint32_t* bm[2];     // queued-in-this-round marks of the next near queue
    int32_t* far[2];
    uint32_t* fbm;       // in-the-pile marks
    int64_t nwords;
    Chunk* chunks;
};

// dist[v] = min(dist[v], d); true when d was smaller than the old value
__device__ __forceinline__ bool atomic_min_improves(float* p, float d) {
    // order-preserving on the bit patterns: non-negative floats order as
    // ints, negative ones in reverse as unsigned ints
    if (d >= 0.0f) return __int_as_float(atomicMin((int*)p, __float_as_int(d))) > d;
    return __uint_as_float(atomicMax((unsigned*)p, __float_as_uint(d))) > d;
}
__device__ __forceinline__ bool atomic_min_improves(int32_t* p, int32_t d) { return atomicMin(p, d) > d; }

__device__ __forceinline__ bool test_and_set(uint32_t* bm, int32_t v) {
    const uint32_t bit = 1u << (v & 31);
    return !(atomicOr(bm + (v >> 5), bit) & bit);
}

template <typename T>
struct SsspRelax {
    using V = T;
    const int32_t* col;
    const T* w;
    T* dist;
    int32_t* qn;
    uint32_t* bn;
    int32_t* ncount;
    int32_t* far;
    uint32_t* fbm;
    int32_t* farcount;
    T thr;
    bool use_far;

    __device__ V load(int32_t u) const { return __ldcg(dist + u); }
    __device__ __forceinline__ void edge(bool valid, V du, int32_t e) {
        int32_t v = -1;
        bool near = false, pile = false;
        if (valid) {
            v = col[e];
            const T nd = elem_add(du, w[e]);
            if (nd < __ldcg(dist + v) && atomic_min_improves(dist + v, nd)) {
                if (!use_far || nd < thr)
                    near = test_and_set(bn, v);  // queued once per round
                else
                    pile = test_and_set(fbm, v);  // in the pile once
            }
        }
        queue_append(near, v, qn, ncount);
        queue_append(pile, v, far, farcount);
    }
};

template <typename T>
__device__ __forceinline__ SsspRelax<T> sssp_relax(const Sssp1Bufs<T>& b, Sssp1State<T>* st) {
    return SsspRelax<T>{b.col,           b.w, b.dist, b.q[st->cur ^ 1], b.bm[st->round & 1], &st->ncount,
                        b.far[st->fcur], b.fbm, &st->farcount, st->thr, st->use_far != 0};
}

template <typename T>
__device__ __forceinline__ void atomic_min_value(T* p, T v) {
    atomic_min_improves(p, v);
}

template <typename T>
__global__ void __launch_bounds__(kT) k_sssp1_light(Sssp1Bufs<T> b, Sssp1State<T>* st) {
    uint32_t* bz = b.bm[(st->round + 1) & 1];  // next round's marks, cleared now
    const int64_t tid = (int64_t)blockIdx.x * kT + threadIdx.x, nth = (int64_t)gridDim.x * kT;
    for (int64_t i = tid; i < b.nwords; i += nth) bz[i] = 0;
    if (st->mode == 0) {
        SsspRelax<T> op = sssp_relax(b, st);
        expand_light(b.q[st->cur], st->fcount, b.rp, b.chunks, &st->nchunks, op);
        return;
    }
    // split: the pile's vertices below the old threshold were expanded as
    // near ones already; below the new one they join the near queue; the
    // rest stay in the pile
    const int32_t* fp = b.far[st->fcur];
    int32_t* fk = b.far[st->fcur ^ 1];
    int32_t* qn = b.q[st->cur ^ 1];
    const int32_t fc = st->farcount;
    const T lo = st->thr_prev, hi = st->thr;
    T kmin = Lim<T>::max();
    const int64_t nr = ((int64_t)fc + 31) / 32 * 32;
    for (int64_t k = tid; k < nr; k += nth) {
        const int32_t v = k < fc ? fp[k] : -1;
        bool near = false, keep = false;
        if (v >= 0) {
            const T d = __ldcg(b.dist + v);
            if (d < lo) {
                atomicAnd(b.fbm + (v >> 5), ~(1u << (v & 31)));
            } else if (d < hi) {
                atomicAnd(b.fbm + (v >> 5), ~(1u << (v & 31)));
                near = true;
            } else {
                keep = true;
                kmin = d < kmin ? d : kmin;
            }
        }
        queue_append(near, v, qn, &st->ncount);
        queue_append(keep, v, fk, &st->farnext);
    }
    if (kmin < Lim<T>::max()) atomic_min_value(&st->far_min, kmin);
}

template <typename T>
__global__ void __launch_bounds__(kT) k_sssp1_heavy(Sssp1Bufs<T> b, Sssp1State<T>* st) {
    if (st->mode != 0) return;
    SsspRelax<T> op = sssp_relax(b, st);
    expand_heavy(b.chunks, st->nchunks, b.rp, op);
}

template <typename T>
__global__ void k_sssp1_control(Sssp1State<T>* st, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    if (st->mode == 1) {  // a split ended: the kept vertices are the pile
        st->farcount = st->farnext;
        st->farnext = 0;
        st->fcur ^= 1;
    }
    const int32_t nc = st->ncount;
    bool cont = st->round < st->max_rounds;
    if (nc > 0) {
        st->mode = 0;
        st->fcount = nc;
        st->cur ^= 1;
    } else if (st->farcount > 0) {
        // the near queue ran dry: raise the threshold past the smallest
        // distance in the pile (known after a split) and split
        const T base = st->mode == 1 ? st->far_min : st->thr;
        st->thr_prev = st->thr;
        const T t = elem_add(base, st->delta);  // saturates for int32
        st->thr = t > base ? t : Lim<T>::max();
        st->mode = 1;
        st->far_min = Lim<T>::max();
    } else {
        cont = false;
    }
    if (cont) st->round += 1;
    st->ncount = 0;
    st->nchunks = 0;
    st->cont = cont ? 1 : 0;
    if (h) cudaGraphSetConditional(h, cont ? 1u : 0u);
}

template <typename T>
__global__ void k_sssp1_init(Sssp1Bufs<T> b, Sssp1State<T>* st, int32_t src, T delta, int use_far) {
    const int64_t tid = (int64_t)blockIdx.x * kT + threadIdx.x, nth = (int64_t)gridDim.x * kT;
    for (int64_t i = tid; i < b.n; i += nth) b.dist[i] = i == src ? T(0) : Lim<T>::max();
    for (int64_t i = tid; i < b.nwords; i += nth) {
        b.bm[0][i] = 0;
        b.bm[1][i] = 0;
        b.fbm[i] = 0;
    }
    if (tid == 0) {
        b.q[0][0] = src;
        st->round = 1;
        st->cur = 0;
        st->fcount = 1;
        st->ncount = 0;
        st->max_rounds = b.n < (int64_t)INT32_MAX / 2 ? 2 * (int32_t)b.n + 1 : INT32_MAX;
        st->nchunks = 0;
        st->mode = 0;
        st->fcur = 0;
        st->farcount = 0;
        st->farnext = 0;
        st->use_far = use_far;
        st->delta = delta;
        st->thr = delta;
        st->thr_prev = T(0);
        st->far_min = Lim<T>::max();
    }
}

// Mean of up to 65536 evenly spaced entries of w (one block).
template <typename T>
__global__ void __launch_bounds__(1024) k_sample_mean(const T* __restrict__ w, int64_t nnz, double* out) {
    __shared__ double red[32];
    const int64_t m = nnz < 65536 ? nnz : 65536;
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < m; k += 1024) s += (double)w[k * nnz / m];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kAll, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = red[threadIdx.x];
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kAll, s, o);
        if (threadIdx.x == 0) *out = m > 0 ? s / (double)m : 0.0;
    }
}

template <typename T>
int run_sssp1(gbk_matrix A, int32_t source, double delta, T* dist, int32_t* rounds, cudaStream_t s) {
    const int64_t n = A->csr.nrows, nnz = A->csr.nnz;
    SingleCache& C = single_cache(A);
    CachedLoop& L = C.sssp;
    const int64_t nwords = (n + 31) / 32;
    const size_t st_b = 256, q_b = 4 * (size_t)n, bm_b = 4 * (size_t)nwords, d_b = sizeof(T) * (size_t)n,
                 ch_b = sizeof(Chunk) * (size_t)max_chunks(nnz);
    int rc = loop_scratch(L, st_b + ch_b + 4 * q_b + 3 * bm_b + d_b);
    if (rc) return rc;
    Sssp1Bufs<T> b{};
    b.rp = A->csr.ptr;
    b.col = A->csr.idx;
    b.w = (const T*)A->csr.val;
    b.n = n;
    b.nwords = nwords;
    char* m = (char*)L.mem;
    Sssp1State<T>* st = (Sssp1State<T>*)m;
    b.chunks = (Chunk*)(m + st_b);
    m += st_b + ch_b;
    b.q[0] = (int32_t*)m;
    b.q[1] = (int32_t*)(m + q_b);
    b.far[0] = (int32_t*)(m + 2 * q_b);
    b.far[1] = (int32_t*)(m + 3 * q_b);
    b.bm[0] = (uint32_t*)(m + 4 * q_b);
    b.bm[1] = (uint32_t*)(m + 4 * q_b + bm_b);
    b.fbm = (uint32_t*)(m + 4 * q_b + 2 * bm_b);
    b.dist = (T*)(m + 4 * q_b + 3 * bm_b);  // 4-byte aligned: every part above is a multiple of 4 bytes
    auto fail = [&](cudaError_t e, const char* what) {
        if (rc == GBK_SUCCESS && e != cudaSuccess) rc = cuda_fail(e, what, __FILE__, __LINE__);
    };
    if (delta == 0.0 && nnz > 0 && C.mean_weight < 0.0) {
        double* mean = (double*)st;  // the state is written after this
        k_sample_mean<T><<<1, 1024, 0, s>>>(b.w, nnz, mean);
        count_launch(1);
        double h = 0.0;
        fail(cudaMemcpyAsync(&h, mean, sizeof(h), cudaMemcpyDeviceToHost, s), "SSSP weight sample");
        fail(cudaStreamSynchronize(s), "SSSP weight sample");
        C.mean_weight = h;
    }
    if (delta == 0.0) {
        // 8 x mean weight / mean row length (R-MAT scale 23 with weights in
        // [1, 255]: 10.1 ms at 8x, 10.8 ms at 32x, 11.4 ms without the pile)
        const double h = C.mean_weight;
        delta = nnz > 0 && h > 0.0 ? 8.0 * h * (double)n / (double)nnz : -1.0;
    }
    const bool use_far = delta > 0.0;
    T dl = T(1);
    if (use_far) {
        if (std::is_integral<T>::value)
            dl = (T)std::min(std::max(delta, 1.0), (double)INT32_MAX / 2);
        else
            dl = (T)std::min(delta, 1e30);
    }
    const int grid = blocks_for_sm((const void*)k_sssp1_light<T>);
    if (rc == GBK_SUCCESS) {
        k_sssp1_init<T><<<grid, kT, 0, s>>>(b, st, source, dl, use_far ? 1 : 0);
        fail(cudaGetLastError(), "k_sssp1_init");
        count_launch(1);
    }
    if (rc == GBK_SUCCESS)
        rc = launch_loop(L, 0, s, &st->cont, [&](cudaStream_t cs, cudaGraphConditionalHandle h) {
            k_sssp1_light<T><<<grid, kT, 0, cs>>>(b, st);
            k_sssp1_heavy<T><<<grid, kT, 0, cs>>>(b, st);
            k_sssp1_control<T><<<1, 32, 0, cs>>>(st, h);
        });
    if (rc == GBK_SUCCESS) fail(cudaMemcpyAsync(dist, b.dist, d_b, cudaMemcpyDeviceToDevice, s), "SSSP distances");
    if (rc == GBK_SUCCESS && rounds) {
        Sssp1State<T> h{};
        fail(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s), "SSSP rounds");
        fail(cudaStreamSynchronize(s), "SSSP rounds");
        *rounds = h.round;
    }
    return rc;
}

// ---- PageRank ---------------------------------------------------------------

struct PrState {
    int32_t iters;
    int32_t itermax;
    int32_t cur;       // which rank buffer holds the current ranks
    int32_t cont;
    float tol;
    float scaled;      // (1 - damping) / n
    float d_over_n;    // damping / n
    float sink;        // sum of the current ranks over the sinks
    float rdiff;       // sum |old - new| of the last iteration
    float damping;
    float inv_damping; // 1 / damping
};

struct PrBufs {
    int64_t n;
    const int32_t* deg;  // entries per column of A
    float* r[2];
    float* w;            // r ./ d, the SpMV input
    float* y;            // A w
    float* part_sink;    // per-block partial sums
    float* part_diff;
    int64_t nsinks;      // columns without entries
    int sparse_sink;     // 1: the sink mass is the sum of the first nsinks ranks
};

// The sink mass as the reference forms it: its sink vector, built by a
// masked assign, turns sparse when it holds at most 0.3 n entries, and its
// masked assign from a sparse mask then reads the ranks at the mask-list
// positions 0 .. nsinks - 1 instead of at the sinks' ids
// (src/backend/operations/generic_operations.h:28-34 with operations.h:63-65).
__device__ __forceinline__ bool pr_sink_term(const PrBufs& b, int64_t i, int32_t deg) {
    return b.sparse_sink ? i < b.nsinks : deg == 0;
}

// d = max(deg / damping, 1 / damping), in float as the reference computes it
__device__ __forceinline__ float pr_d(float damping, float inv_damping, int32_t deg) {
    return fmaxf((float)deg / damping, inv_damping);
}

template <int NT>
__device__ __forceinline__ float block_sum(float v) {
    __shared__ float red[NT / 32];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kAll, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.0f;
    if (threadIdx.x < 32) {
        t = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0f;
        for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(kAll, t, o);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

// r0 = 1 / n, w = r0 ./ d, partial sums of r0 over the sinks
__global__ void __launch_bounds__(kT) k_pr_init(PrBufs b, const PrState* st, float r0) {
    const float dmp = st->damping, inv = st->inv_damping;
    float sink = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < b.n; i += (int64_t)gridDim.x * kT) {
        const int32_t dg = b.deg[i];
        b.r[0][i] = r0;
        b.w[i] = r0 / pr_d(dmp, inv, dg);
        if (pr_sink_term(b, i, dg)) sink += r0;
    }
    sink = block_sum<kT>(sink);
    if (threadIdx.x == 0) {
        b.part_sink[blockIdx.x] = sink;
        b.part_diff[blockIdx.x] = 0.0f;
    }
}

// r_new = teleport + y with teleport = (1 - damping) / n + damping / n * (sum of
// the old ranks over the sinks); partial sums of |r_old - r_new| and of the
// new ranks over the sinks; w = r_new ./ d for the next product
__global__ void __launch_bounds__(kT) k_pr_post(PrBufs b, const PrState* st) {
    const float teleport = st->scaled + st->d_over_n * st->sink;
    const float dmp = st->damping, inv = st->inv_damping;
    const float* __restrict__ ro = b.r[st->cur];
    float* __restrict__ rn = b.r[st->cur ^ 1];
    float sink = 0.0f, diff = 0.0f;
    for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < b.n; i += (int64_t)gridDim.x * kT) {
        const int32_t dg = b.deg[i];
        const float r = teleport + b.y[i];
        diff += fabsf(ro[i] - r);
        rn[i] = r;
        b.w[i] = r / pr_d(dmp, inv, dg);
        if (pr_sink_term(b, i, dg)) sink += r;
    }
    sink = block_sum<kT>(sink);
    diff = block_sum<kT>(diff);
    if (threadIdx.x == 0) {
        b.part_sink[blockIdx.x] = sink;
        b.part_diff[blockIdx.x] = diff;
    }
}

// Sums the partials in a fixed order (the same result every run), counts
// the iteration (iter = 1) and decides whether another one runs.
__global__ void __launch_bounds__(256) k_pr_control(PrBufs b, PrState* st, int nparts, int iter,
                                                    cudaGraphConditionalHandle h) {
    float s = 0.0f, d = 0.0f;
    for (int i = threadIdx.x; i < nparts; i += 256) {
        s += b.part_sink[i];
        d += b.part_diff[i];
    }
    s = block_sum<256>(s);
    d = block_sum<256>(d);
    if (threadIdx.x == 0) {
        st->sink = s;
        if (iter) {
            st->rdiff = d;
            st->iters += 1;
            st->cur ^= 1;
        }
        const bool cont = st->iters < st->itermax && !(st->tol > 0.0f && st->rdiff < st->tol);
        st->cont = cont ? 1 : 0;
        if (h) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

__global__ void k_col_degree(const int32_t* __restrict__ col, int64_t nnz, int32_t* deg) {
    for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * kT)
        atomicAdd(deg + col[i], 1);
}

__global__ void k_count_zero(const int32_t* __restrict__ deg, int64_t n, unsigned long long* count) {
    unsigned c = 0;
    for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT) c += deg[i] == 0;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(kAll, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// ---- CC ---------------------------------------------------------------------

__device__ __forceinline__ int32_t uf_find(int32_t* p, int32_t x) {
    // path halving; a vertex only ever moves to a smaller root
    int32_t px = __ldcg(p + x);
    while (px != x) {
        const int32_t ppx = __ldcg(p + px);
        if (ppx != px) p[x] = ppx;
        x = px;
        px = ppx;
    }
    return x;
}

__device__ __forceinline__ void uf_unite(int32_t* p, int32_t a, int32_t b) {
    for (;;) {
        a = uf_find(p, a);
        b = uf_find(p, b);
        if (a == b) return;
        if (a < b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        // link the larger root a under the smaller root b
        if (atomicCAS(p + a, a, b) == a) return;
    }
}

__global__ void k_cc_init(int32_t* p, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
    if (i < n) p[i] = (int32_t)i;
}

// Every vertex links along its entry r (r = 0, 1).
__global__ void k_cc_link_entry(const int32_t* __restrict__ rp, const int32_t* __restrict__ col, int64_t n,
                                int32_t* p, int r) {
    const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
    if (i >= n) return;
    const int32_t u = (int32_t)i, beg = rp[u];
    if (rp[u + 1] - beg > r) {
        const int32_t v = col[beg + r];
        if (v != u) uf_unite(p, u, v);
    }
}

__global__ void k_cc_compress(int32_t* p, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
    if (i < n) p[i] = uf_find(p, (int32_t)i);
}

// The most frequent root among 1024 sampled vertices (ties: the smaller
// root), one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_cc_sample_mode(int32_t* p, int64_t n, int32_t* mode) {
    __shared__ int32_t roots[1024];
    __shared__ unsigned long long best;
    const int i = threadIdx.x;
    const uint64_t h = (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull;
    roots[i] = uf_find(p, (int32_t)((h >> 20) % (uint64_t)n));
    if (i == 0) best = 0;
    __syncthreads();
    const int32_t mine = roots[i];
    uint32_t count = 0;
    for (int k = 0; k < 1024; ++k) count += roots[k] == mine;
    atomicMax(&best, ((unsigned long long)count << 32) | (uint32_t)(INT32_MAX - mine));
    __syncthreads();
    if (i == 0) *mode = INT32_MAX - (int32_t)(uint32_t)(best & 0xffffffffu);
}

// Vertices outside the sampled component (every vertex when skip == 0) link
// along their entries from the third on: rows under kHeavy entries by their
// lane, longer ones by the whole warp.
__global__ void __launch_bounds__(kT) k_cc_link_rest(const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                                     int64_t n, int32_t* p, const int32_t* mode, int skip) {
    const int lane = threadIdx.x & 31;
    const int32_t c = skip ? *mode : -1;
    const int64_t tid = (int64_t)blockIdx.x * kT + threadIdx.x, nth = (int64_t)gridDim.x * kT;
    const int64_t nr = (n + 31) / 32 * 32;
    for (int64_t u0 = tid; u0 < nr; u0 += nth) {
        const int32_t u = (int32_t)u0;
        // after the compression every member of the sampled component points at its root
        const bool act = u0 < n && __ldcg(p + u) != c;
        const int32_t beg = act ? rp[u] + 2 : 0, deg = act ? max(rp[u + 1] - beg, 0) : 0;
        if (deg < kHeavy)
            for (int32_t e = beg; e < beg + deg; ++e) {
                const int32_t v = col[e];
                if (v != u) uf_unite(p, u, v);
            }
        unsigned hubs = __ballot_sync(kAll, deg >= kHeavy);
        while (hubs) {
            const int h = __ffs(hubs) - 1;
            hubs &= hubs - 1;
            const int32_t hu = __shfl_sync(kAll, u, h), hb = __shfl_sync(kAll, beg, h),
                          hd = __shfl_sync(kAll, deg, h);
            for (int32_t e = lane; e < hd; e += 32) {
                const int32_t v = col[hb + e];
                if (v != hu) uf_unite(p, hu, v);
            }
        }
    }
}

template <typename T>
__global__ void k_cc_labels(int32_t* p, int64_t n, T* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
    if (i < n) out[i] = (T)uf_find(p, (int32_t)i);
}

// The CSC lists every column's rows in ascending order; the pattern is
// symmetric exactly when it equals the CSR, whose rows are then sorted too.
__global__ void k_same_pattern(const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                               const int32_t* __restrict__ cp, const int32_t* __restrict__ row, int64_t n,
                               int64_t nnz, int32_t* diff) {
    const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
    bool d = (i <= n && rp[i] != cp[i]) || (i < nnz && col[i] != row[i]);
    if (__any_sync(kAll, d) && (threadIdx.x & 31) == 0) atomicOr(diff, 1);
}

int pattern_symmetric(gbk_matrix A, cudaStream_t s, bool* out) {
    if (A->pattern_symmetric < 0) {
        const int64_t n = A->csr.nrows;
        if (A->csr.ncols != n) {
            A->pattern_symmetric = 0;
        } else {
            int rc = ensure_csc(A, s);
            if (rc) return rc;
            int32_t* diff = nullptr;
            GBK_CUDA(cudaMallocAsync((void**)&diff, 4, s));
            GBK_CUDA(cudaMemsetAsync(diff, 0, 4, s));
            const int64_t cnt = std::max<int64_t>(n + 1, A->csr.nnz);
            k_same_pattern<<<grid1(cnt), kT, 0, s>>>(A->csr.ptr, A->csr.idx, A->csc.ptr, A->csc.idx, n,
                                                      A->csr.nnz, diff);
            GBK_LAUNCHED();
            int32_t h = 1;
            cudaError_t e = cudaMemcpyAsync(&h, diff, 4, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            cudaFreeAsync(diff, s);
            if (e != cudaSuccess) return cuda_fail(e, "pattern symmetry check", __FILE__, __LINE__);
            A->pattern_symmetric = h == 0 ? 1 : 0;
        }
    }
    *out = A->pattern_symmetric == 1;
    return GBK_SUCCESS;
}

}  // namespace

}  // namespace gbk

using namespace gbk;

extern "C" int gbk_bfs_levels(gbk_matrix A, int64_t source, int direction, gbk_dtype level_type, void* levels,
                              int32_t* depth, void* stream) {
    GBK_REQUIRE(A && levels, GBK_NULL_POINTER, "gbk_bfs_levels: NULL argument");
    const int64_t n = A->csr.nrows;
    GBK_REQUIRE(A->csr.ncols == n, GBK_DIMENSION_MISMATCH, "gbk_bfs_levels: the matrix must be square");
    GBK_REQUIRE(source >= 0 && source < n, GBK_INVALID_INDEX, "gbk_bfs_levels: source %lld outside [0, %lld)",
                (long long)source, (long long)n);
    GBK_REQUIRE(direction >= 0 && direction <= 2, GBK_INVALID_VALUE, "gbk_bfs_levels: direction %d", direction);
    GBK_REQUIRE(level_type == GBK_F32 || level_type == GBK_I32 || level_type == GBK_F64 || level_type == GBK_I64,
                GBK_INVALID_VALUE, "gbk_bfs_levels: level type %d", (int)level_type);
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ensure_csc(A, s);
    if (rc) return rc;
    CachedLoop& L = single_cache(A).bfs;
    const size_t st_b = 256, lv_b = 4 * (size_t)n, q_b = 4 * (size_t)n, bm_b = 4 * (size_t)((n + 31) / 32),
                 ch_b = sizeof(Chunk) * (size_t)max_chunks(A->csr.nnz);
    rc = loop_scratch(L, st_b + ch_b + lv_b + 2 * q_b + 3 * bm_b);
    if (rc) return rc;
    Bfs1Bufs b{};
    b.rp = A->csr.ptr;
    b.col = A->csr.idx;
    b.crp = A->csc.ptr;
    b.crow = A->csc.idx;
    b.n = n;
    b.nwords = (n + 31) / 32;
    char* m = (char*)L.mem;
    Bfs1State* st = (Bfs1State*)m;
    b.chunks = (Chunk*)(m + st_b);
    m += st_b + ch_b;
    b.lv = (int32_t*)m;
    b.q[0] = (int32_t*)(m + lv_b);
    b.q[1] = (int32_t*)(m + lv_b + q_b);
    for (int k = 0; k < 3; ++k) b.bm[k] = (uint32_t*)(m + lv_b + 2 * q_b + k * bm_b);
    const int grid = blocks_for_sm((const void*)k_bfs1_light);
    k_bfs1_init<<<grid, kT, 0, s>>>(b, st, (int32_t)source, (long long)A->csr.nnz, 14, 24, direction);
    cudaError_t e = cudaGetLastError();
    rc = e == cudaSuccess ? GBK_SUCCESS : cuda_fail(e, "k_bfs1_init", __FILE__, __LINE__);
    count_launch(1);
    if (rc == GBK_SUCCESS)
        rc = launch_loop(L, 0, s, &st->cont, [&](cudaStream_t cs, cudaGraphConditionalHandle h) {
            k_bfs1_light<<<grid, kT, 0, cs>>>(b, st);
            k_bfs1_heavy<<<grid, kT, 0, cs>>>(b, st);
            k_bfs1_control<<<1, 32, 0, cs>>>(st, b.n, h);
        });
    if (rc == GBK_SUCCESS) {
        // the levels into the caller's array in its type
#define LV_OUT(TY) k_levels_out<TY><<<grid1(n), kT, 0, s>>>(b.lv, n, (TY*)levels)
        switch (level_type) {
            case GBK_F32: LV_OUT(float); break;
            case GBK_F64: LV_OUT(double); break;
            case GBK_I32: LV_OUT(int32_t); break;
            default: LV_OUT(int64_t); break;
        }
#undef LV_OUT
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "level conversion", __FILE__, __LINE__);
        count_launch(1);
    }
    if (rc == GBK_SUCCESS && depth) {
        Bfs1State h{};
        e = cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "BFS depth", __FILE__, __LINE__);
        *depth = h.level;
    }
    return rc;
}

extern "C" int gbk_sssp_dist(gbk_matrix A, int64_t source, double delta, void* dist, int32_t* rounds,
                             void* stream) {
    GBK_REQUIRE(A && dist, GBK_NULL_POINTER, "gbk_sssp_dist: NULL argument");
    const int64_t n = A->csr.nrows;
    GBK_REQUIRE(A->csr.ncols == n, GBK_DIMENSION_MISMATCH, "gbk_sssp_dist: the matrix must be square");
    GBK_REQUIRE(source >= 0 && source < n, GBK_INVALID_INDEX, "gbk_sssp_dist: source %lld outside [0, %lld)",
                (long long)source, (long long)n);
    cudaStream_t s = (cudaStream_t)stream;
    if (A->vtype == GBK_F32) return run_sssp1<float>(A, (int32_t)source, delta, (float*)dist, rounds, s);
    return run_sssp1<int32_t>(A, (int32_t)source, delta, (int32_t*)dist, rounds, s);
}

extern "C" int gbk_pagerank(gbk_matrix A, int32_t itermax, double damping, double tol, float* ranks,
                            int32_t* iters, float* rdiff, void* stream) {
    GBK_REQUIRE(A && ranks, GBK_NULL_POINTER, "gbk_pagerank: NULL argument");
    const int64_t n = A->csr.nrows;
    GBK_REQUIRE(A->csr.ncols == n, GBK_DIMENSION_MISMATCH, "gbk_pagerank: the matrix must be square");
    GBK_REQUIRE(A->vtype == GBK_F32, GBK_DOMAIN_MISMATCH, "gbk_pagerank: the matrix values must be GBK_F32");
    GBK_REQUIRE(damping > 0.0, GBK_INVALID_VALUE, "gbk_pagerank: damping %g must be positive", damping);
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        if (iters) *iters = 0;
        return GBK_SUCCESS;
    }
    if (!A->coldeg) {
        int32_t* deg = nullptr;
        GBK_CUDA(cudaMalloc((void**)&deg, 4 * (size_t)n + 16));
        unsigned long long* zero = (unsigned long long*)(deg + ((n + 1) / 2) * 2);
        GBK_CUDA(cudaMemsetAsync(deg, 0, 4 * (size_t)n + 16, s));
        const unsigned g = (unsigned)std::min<int64_t>(grid1(std::max(n, A->csr.nnz)), 8 * num_sms());
        if (A->csr.nnz > 0) {
            k_col_degree<<<g, kT, 0, s>>>(A->csr.idx, A->csr.nnz, deg);
            GBK_LAUNCHED();
        }
        k_count_zero<<<g, kT, 0, s>>>(deg, n, zero);
        GBK_LAUNCHED();
        unsigned long long hz = 0;
        GBK_CUDA(cudaMemcpyAsync(&hz, zero, 8, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        A->coldeg = deg;
        A->coldeg_zero = (int64_t)hz;
    }
    const int nb = blocks_for_sm((const void*)k_pr_post);
    CachedLoop& L = single_cache(A).pr;
    const size_t st_b = 256, v_b = 4 * (size_t)n, p_b = 4 * (size_t)nb;
    int rc = loop_scratch(L, st_b + 4 * v_b + 2 * p_b);
    if (rc) return rc;
    PrBufs b{};
    b.n = n;
    b.deg = A->coldeg;
    b.nsinks = A->coldeg_zero;
    b.sparse_sink = A->coldeg_zero <= (int64_t)((double)n * 0.3) ? 1 : 0;
    char* m = (char*)L.mem;
    PrState* st = (PrState*)m;
    m += st_b;
    b.r[0] = (float*)m;
    b.r[1] = (float*)(m + v_b);
    b.w = (float*)(m + 2 * v_b);
    b.y = (float*)(m + 3 * v_b);
    b.part_sink = (float*)(m + 4 * v_b);
    b.part_diff = (float*)(m + 4 * v_b + p_b);
    PrState h0{};
    h0.itermax = itermax;
    h0.tol = (float)tol;
    h0.scaled = (float)((1.0 - damping) / (double)n);
    h0.d_over_n = (float)(damping / (double)n);
    h0.rdiff = 1.0f;
    h0.damping = (float)damping;
    h0.inv_damping = (float)(1.0 / damping);
    auto fail = [&](cudaError_t e, const char* what) {
        if (rc == GBK_SUCCESS && e != cudaSuccess) rc = cuda_fail(e, what, __FILE__, __LINE__);
    };
    fail(cudaMemcpyAsync(st, &h0, sizeof(h0), cudaMemcpyHostToDevice, s), "gbk_pagerank state");
    if (rc == GBK_SUCCESS) {
        k_pr_init<<<nb, kT, 0, s>>>(b, st, (float)(1.0 / (double)n));
        k_pr_control<<<1, 256, 0, s>>>(b, st, nb, 0, 0);
        fail(cudaGetLastError(), "k_pr_init");
        count_launch(2);
    }
    auto iterate = [&](cudaStream_t cs, cudaGraphConditionalHandle hd) {
        int r = gbk_mxv(A, 0, GBK_PLUS_SECOND, GBK_OP_SECOND, GBK_F32, b.w, b.y, nullptr, GBK_F32, GBK_MASK_DEFAULT,
                        cs);
        k_pr_post<<<nb, kT, 0, cs>>>(b, st);
        k_pr_control<<<1, 256, 0, cs>>>(b, st, nb, 1, hd);
        count_launch(2);
        return r;
    };
    PrState h{};
    h.cont = itermax > 0 && !(tol > 0.0 && 1.0f < (float)tol) ? 1 : 0;
    // The graph captures the SpMV of the matrix's current format; a new format
    // (its generation) rebuilds it.  Before the first capture one iteration
    // runs outside the graph: the first product also builds whatever the
    // format builds on first use.
    const bool cached = L.exec && L.key == A->format_gen && !host_loop_mode();
    if (rc == GBK_SUCCESS && h.cont && !cached) {
        rc = iterate(s, 0);
        fail(cudaGetLastError(), "PageRank iteration");
        fail(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s), "gbk_pagerank state");
        fail(cudaStreamSynchronize(s), "gbk_pagerank state");
    }
    if (rc == GBK_SUCCESS && h.cont) {
        int irc = GBK_SUCCESS;
        rc = launch_loop(L, A->format_gen, s, &st->cont,
                         [&](cudaStream_t cs, cudaGraphConditionalHandle hd) { irc = iterate(cs, hd); });
        if (rc == GBK_SUCCESS) rc = irc;
    }
    if (rc == GBK_SUCCESS) {
        fail(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s), "gbk_pagerank state");
        fail(cudaStreamSynchronize(s), "gbk_pagerank state");
    }
    if (rc == GBK_SUCCESS)
        fail(cudaMemcpyAsync(ranks, b.r[h.cur & 1], v_b, cudaMemcpyDeviceToDevice, s), "gbk_pagerank ranks");
    if (rc == GBK_SUCCESS) {
        if (iters) *iters = h.iters;
        if (rdiff) *rdiff = h.rdiff;
    }
    return rc;
}

extern "C" int gbk_matrix_pattern_symmetric(gbk_matrix A, int32_t* symmetric, void* stream) {
    GBK_REQUIRE(A && symmetric, GBK_NULL_POINTER, "gbk_matrix_pattern_symmetric: NULL argument");
    bool sym = false;
    int rc = pattern_symmetric(A, (cudaStream_t)stream, &sym);
    if (rc) return rc;
    *symmetric = sym ? 1 : 0;
    return GBK_SUCCESS;
}

extern "C" int gbk_cc_labels(gbk_matrix A, gbk_dtype label_type, void* labels, void* stream) {
    GBK_REQUIRE(A && labels, GBK_NULL_POINTER, "gbk_cc_labels: NULL argument");
    const int64_t n = A->csr.nrows;
    GBK_REQUIRE(A->csr.ncols == n, GBK_DIMENSION_MISMATCH, "gbk_cc_labels: the matrix must be square");
    GBK_REQUIRE(label_type == GBK_F32 || label_type == GBK_I32 || label_type == GBK_I64, GBK_INVALID_VALUE,
                "gbk_cc_labels: label type %d", (int)label_type);
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return GBK_SUCCESS;
    bool sym = false;
    int rc = pattern_symmetric(A, s, &sym);
    if (rc) return rc;
    // int32 labels: the forest lives in the output itself
    const bool direct = label_type == GBK_I32;
    int32_t* p = (int32_t*)labels;
    int32_t* mode = nullptr;
    GBK_CUDA(cudaMallocAsync((void**)&mode, direct ? 16 : 16 + 4 * (size_t)n, s));
    if (!direct) p = mode + 4;
    const unsigned g = grid1(n);
    k_cc_init<<<g, kT, 0, s>>>(p, n);
    for (int r = 0; r < 2; ++r) {
        k_cc_link_entry<<<g, kT, 0, s>>>(A->csr.ptr, A->csr.idx, n, p, r);
        k_cc_compress<<<g, kT, 0, s>>>(p, n);
    }
    k_cc_sample_mode<<<1, 1024, 0, s>>>(p, n, mode);
    k_cc_link_rest<<<blocks_for_sm((const void*)k_cc_link_rest), kT, 0, s>>>(A->csr.ptr, A->csr.idx, n, p, mode,
                                                                              sym ? 1 : 0);
    switch (label_type) {
        case GBK_F32: k_cc_labels<float><<<g, kT, 0, s>>>(p, n, (float*)labels); break;
        case GBK_I32: k_cc_compress<<<g, kT, 0, s>>>(p, n); break;
        default: k_cc_labels<int64_t><<<g, kT, 0, s>>>(p, n, (int64_t*)labels); break;
    }
    count_launch(8);
    // a failed launch leaves its error for this check; the scratch goes back either way
    const cudaError_t e = cudaGetLastError();
    cudaFreeAsync(mode, s);
    if (e != cudaSuccess) return cuda_fail(e, "gbk_cc_labels launch", __FILE__, __LINE__);
    return GBK_SUCCESS;
}
