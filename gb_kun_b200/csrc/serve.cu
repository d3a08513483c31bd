// Continuous-batching query server over one resident graph (host runtime).
//
// Each batch (batched.h) owns a CUDA stream and cycles through
//   [summaries + copies of the lanes that finished] -> [release those lanes]
//   -> [admit waiting queries into free lanes] -> [graph launch: a few
//   iterations, stopping early when a lane finishes] -> [status to the host]
// and the host loop polls every batch's event without blocking, so batches
// of different kinds run concurrently and a request never waits for the
// requests ahead of it to finish.  Admission is by device memory: a batch is
// created only when its state fits the budget, and with keep_results each
// admitted query reserves its result vector first.  The reference serves no
// queries; its drivers run one algorithm per process (bfs.cpp, sssp.cpp).
#include <chrono>
#include <deque>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batched.h"
#include "common.cuh"
#include "gbk_serve.h"

namespace gbk {
namespace {

using Clock = std::chrono::steady_clock;

struct Slot {
    int kind = 0;
    int index = 0;
    Batch* b = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    bool inflight = false;
    int lanes_used = 0;
    int it_seen = 0;
    std::vector<int64_t> lane_q;           // query per lane, -1 = free
    std::vector<int64_t> pending_digest;   // queries whose summary copy is in flight
    std::vector<int> pending_lane;
    LaneDigest* d_dig = nullptr;
    LaneDigest* h_dig = nullptr;

    ~Slot() {
        if (s) cudaStreamSynchronize(s);
        delete b;
        cudaFree(d_dig);
        cudaFreeHost(h_dig);
        if (ev) cudaEventDestroy(ev);
        if (s) cudaStreamDestroy(s);
    }
    int free_lanes() const {
        int f = 0;
        for (int l = 0; l < lanes_used; ++l) f += lane_q[l] < 0;
        return f;
    }
    bool busy() const {
        for (int l = 0; l < lanes_used; ++l)
            if (lane_q[l] >= 0) return true;
        return !pending_digest.empty();
    }
};

struct QState {
    int kind = 0;
    int32_t src = 0;
    double t_arr = 0, t_adm = -1, t_done = -1;
    int slot = -1, lane = -1;
    int32_t iters = 0;
    LaneDigest dig{};
    bool done = false;
};

}  // namespace
}  // namespace gbk

struct gbk_server_s {
    gbk_matrix A = nullptr;
    gbk_server_config cfg{};
    gbk::BatchOptions opt;
    int64_t n = 0, nnz = 0;
    int64_t budget = 0, batch_bytes = 0, result_bytes = 0;
    std::vector<gbk::Slot*> slots;
    std::vector<gbk::QState> q;
    std::deque<int64_t> pending[3];
    std::unordered_map<int64_t, void*> results;
    int inflight = 0;
    int64_t ndone = 0;
    gbk::Clock::time_point t0;

    ~gbk_server_s() {
        for (auto* sl : slots) delete sl;
        for (auto& kv : results) cudaFree(kv.second);
    }
    double now() const { return std::chrono::duration<double>(gbk::Clock::now() - t0).count(); }
    int64_t used() const { return batch_bytes + result_bytes; }
};

namespace gbk {
namespace {

constexpr int kKinds = 3;

// Device bytes a new batch of `kind` will hold (checked before creating it).
int64_t batch_estimate(const gbk_server_s* S, int kind) {
    const int64_t n = std::max<int64_t>(S->n, 1), items = S->n + S->nnz / 256 + 1;
    switch (kind) {
        case kBatchBfs: return n * (24 + 4 * kBfsLanes);
        case kBatchPpr: return n * (8 + 4 * 4 * 32) + 12 * items + 128 * (S->nnz / 256 + 1);
        default: return n * (4 * 32 + 8) + 12 * items;
    }
}

int make_slot(gbk_server_s* S, int kind, Slot** out) {
    Slot* sl = new Slot();
    sl->kind = kind;
    sl->index = (int)S->slots.size();
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        delete sl;
        return cuda_fail(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
    }
    sl->s = s;
    // the matrix's tuned options for this kind, with the server's PPR parameters
    BatchOptions o = base_options(S->A, kind);
    o.damping = S->opt.damping;
    o.tol = S->opt.tol;
    o.itermax = S->opt.itermax;
    int rc = kind == kBatchBfs   ? make_bfs_batch(S->A, o, &sl->b, s)
             : kind == kBatchPpr ? make_ppr_batch(S->A, o, &sl->b, s)
                                 : make_sssp_batch(S->A, o, &sl->b, s);
    if (rc) {
        delete sl;
        return rc;
    }
    const int lanes = sl->b->lanes();
    sl->lanes_used = S->cfg.lanes_per_batch > 0 ? std::min(S->cfg.lanes_per_batch, lanes) : lanes;
    sl->lane_q.assign(lanes, -1);
    cudaError_t e = cudaEventCreateWithFlags(&sl->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&sl->d_dig, sizeof(LaneDigest) * lanes);
    if (e == cudaSuccess) e = cudaMallocHost(&sl->h_dig, sizeof(LaneDigest) * lanes);
    if (e != cudaSuccess) {
        delete sl;
        return cuda_fail(e, "server slot set-up", __FILE__, __LINE__);
    }
    S->batch_bytes += (int64_t)sl->b->device_bytes();
    S->slots.push_back(sl);
    *out = sl;
    return GBK_SUCCESS;
}

// One step of a batch whose previous launch has completed (or that is idle):
// collect summaries, retire finished lanes, admit, launch.  *progress tells
// whether anything happened (a completion, an admission or a launch).
int cycle(gbk_server_s* S, Slot* sl, bool* progress) {
    Batch* b = sl->b;
    const int64_t n = S->n;
    *progress = sl->inflight;
    if (sl->inflight) {
        sl->inflight = false;
        const BatchStatus* st = b->host();
        count_launch(b->kernels_per_iter() * (st->iter - sl->it_seen));
        sl->it_seen = st->iter;
        const double t = S->now();
        for (size_t k = 0; k < sl->pending_digest.size(); ++k) {
            QState& q = S->q[sl->pending_digest[k]];
            q.dig = sl->h_dig[sl->pending_lane[k]];
            q.t_done = t;
            q.done = true;
            S->ndone++;
        }
        sl->pending_digest.clear();
        sl->pending_lane.clear();
        unsigned long long fin = 0;
        for (int l = 0; l < sl->lanes_used; ++l)
            if (sl->lane_q[l] >= 0 && ((st->finished >> l) & 1)) fin |= 1ull << l;
        if (fin) {
            int rc = b->digest(fin, sl->d_dig, sl->s);
            if (rc) return rc;
            for (int l = 0; l < sl->lanes_used; ++l) {
                if (!((fin >> l) & 1)) continue;
                const int64_t qi = sl->lane_q[l];
                S->q[qi].iters = st->iters[l];
                if (S->cfg.keep_results) {
                    void* dst = nullptr;
                    GBK_CUDA(cudaMallocAsync(&dst, 4 * (size_t)std::max<int64_t>(n, 1), sl->s));
                    S->results[qi] = dst;
                    rc = b->extract(l, 1, dst, n, sl->s);
                    if (rc) return rc;
                }
                sl->pending_digest.push_back(qi);
                sl->pending_lane.push_back(l);
                sl->lane_q[l] = -1;
                S->inflight--;
            }
            rc = b->release(fin, sl->s);
            if (rc) return rc;
            GBK_CUDA(cudaMemcpyAsync(sl->h_dig, sl->d_dig, sizeof(LaneDigest) * b->lanes(), cudaMemcpyDeviceToHost,
                                     sl->s));
        }
    }
    // admission: free lanes, the in-flight cap and (kept results) memory
    std::deque<int64_t>& pend = S->pending[sl->kind];
    unsigned long long mask = 0;
    int32_t src[64] = {0};
    const double t = S->now();
    const int64_t rbytes = 4 * std::max<int64_t>(n, 1);
    for (int l = 0; l < sl->lanes_used && !pend.empty(); ++l) {
        if (sl->lane_q[l] >= 0) continue;
        if (S->cfg.max_inflight > 0 && S->inflight >= S->cfg.max_inflight) break;
        if (S->cfg.keep_results && S->used() + rbytes > S->budget) break;
        const int64_t qi = pend.front();
        pend.pop_front();
        QState& q = S->q[qi];
        q.t_adm = t;
        q.slot = sl->index;
        q.lane = l;
        sl->lane_q[l] = qi;
        src[l] = q.src;
        mask |= 1ull << l;
        S->inflight++;
        if (S->cfg.keep_results) S->result_bytes += rbytes;
    }
    if (mask) {
        const int rc = b->admit(mask, src, sl->s);
        if (rc) return rc;
        S->batch_bytes = 0;
        for (auto* o : S->slots) S->batch_bytes += (int64_t)o->b->device_bytes();
    }
    bool active = false;
    for (int l = 0; l < sl->lanes_used; ++l) active |= sl->lane_q[l] >= 0;
    if (active) {
        const int budget = S->cfg.max_inflight == 1 ? (1 << 30) : S->cfg.iters_per_launch;
        const int rc = b->launch(budget, true, sl->s);
        if (rc) return rc;
    }
    if (active || !sl->pending_digest.empty()) {
        GBK_CUDA(cudaEventRecord(sl->ev, sl->s));
        sl->inflight = true;
        *progress = true;
    }
    return GBK_SUCCESS;
}

// Creates a batch for `kind` when queries wait, no batch of that kind has a
// free lane, the kind's batch cap allows one and its state fits the budget.
int grow(gbk_server_s* S, int kind, bool* made) {
    *made = false;
    if (S->pending[kind].empty()) return GBK_SUCCESS;
    if (S->cfg.max_inflight > 0 && S->inflight >= S->cfg.max_inflight) return GBK_SUCCESS;
    int count = 0;
    for (auto* sl : S->slots) {
        if (sl->kind != kind) continue;
        count++;
        if (sl->free_lanes() > 0) return GBK_SUCCESS;
    }
    const int cap = S->cfg.max_batches[kind] > 0 ? S->cfg.max_batches[kind] : 1;
    if (count >= cap) return GBK_SUCCESS;
    if (count > 0 && S->used() + batch_estimate(S, kind) > S->budget) return GBK_SUCCESS;
    Slot* sl = nullptr;
    int rc = make_slot(S, kind, &sl);
    if (rc) return rc;
    *made = true;
    bool progress = false;
    return cycle(S, sl, &progress);
}

}  // namespace
}  // namespace gbk

using namespace gbk;

extern "C" {

int gbk_server_create(gbk_matrix A, const gbk_server_config* cfg, gbk_server* out) {
    GBK_REQUIRE(A && out, GBK_NULL_POINTER, "gbk_server_create: NULL argument");
    GBK_REQUIRE(A->csr.nrows == A->csr.ncols, GBK_DIMENSION_MISMATCH, "gbk_server_create: matrix must be square");
    gbk_server S = new gbk_server_s();
    S->A = A;
    if (cfg) S->cfg = *cfg;
    gbk_server_config& c = S->cfg;
    if (c.iters_per_launch <= 0) c.iters_per_launch = 4;
    if (c.ppr_damping <= 0) c.ppr_damping = 0.85;
    if (c.ppr_tol <= 0) c.ppr_tol = 1e-6;
    if (c.ppr_itermax <= 0) c.ppr_itermax = 100;
    if (c.lanes_per_batch < 0 || c.max_inflight < 0) {
        delete S;
        set_error("gbk_server_create: negative lanes_per_batch or max_inflight");
        return GBK_INVALID_VALUE;
    }
    S->opt.damping = (float)c.ppr_damping;
    S->opt.tol = c.ppr_tol;
    S->opt.itermax = c.ppr_itermax;
    S->n = A->csr.nrows;
    S->nnz = A->csr.nnz;
    if (c.memory_budget > 0) {
        S->budget = c.memory_budget;
    } else {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        S->budget = (int64_t)(0.8 * (double)fr);
    }
    *out = S;
    return GBK_SUCCESS;
}

int gbk_server_destroy(gbk_server s) {
    delete s;
    return GBK_SUCCESS;
}

int gbk_server_run_trace(gbk_server S, const int32_t* kinds, const int32_t* sources, const double* arrivals,
                         int64_t nq, gbk_query_result* out, double* wall_s) {
    GBK_REQUIRE(S && (nq == 0 || (kinds && sources && arrivals && out)), GBK_NULL_POINTER,
                "gbk_server_run_trace: NULL argument");
    for (int64_t i = 0; i < nq; ++i) {
        GBK_REQUIRE(kinds[i] >= 0 && kinds[i] < kKinds, GBK_INVALID_VALUE, "gbk_server_run_trace: bad kind %d",
                    kinds[i]);
        GBK_REQUIRE(sources[i] >= 0 && sources[i] < S->n, GBK_INVALID_INDEX,
                    "gbk_server_run_trace: source %d out of range", sources[i]);
        GBK_REQUIRE(i == 0 || arrivals[i] >= arrivals[i - 1], GBK_INVALID_VALUE,
                    "gbk_server_run_trace: arrivals must ascend");
    }
    for (auto& kv : S->results) cudaFree(kv.second);
    S->results.clear();
    S->result_bytes = 0;
    S->q.assign(nq, QState{});
    for (int k = 0; k < kKinds; ++k) S->pending[k].clear();
    S->inflight = 0;
    S->ndone = 0;
    for (int64_t i = 0; i < nq; ++i) {
        S->q[i].kind = kinds[i];
        S->q[i].src = sources[i];
        S->q[i].t_arr = arrivals[i];
    }
    S->t0 = Clock::now();
    int64_t next = 0;
    while (S->ndone < nq) {
        const double t = S->now();
        while (next < nq && arrivals[next] <= t) {
            S->pending[kinds[next]].push_back(next);
            next++;
        }
        bool worked = false;
        for (auto* sl : S->slots) {
            if (sl->inflight) {
                const cudaError_t e = cudaEventQuery(sl->ev);
                if (e == cudaErrorNotReady) continue;
                if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery", __FILE__, __LINE__);
            } else if (!sl->busy() && S->pending[sl->kind].empty()) {
                continue;
            }
            bool progress = false;
            const int rc = cycle(S, sl, &progress);
            if (rc) return rc;
            worked |= progress;
        }
        for (int k = 0; k < kKinds; ++k) {
            bool made = false;
            const int rc = grow(S, k, &made);
            if (rc) return rc;
            worked |= made;
        }
        if (!worked) {
            bool any_inflight = false;
            for (auto* sl : S->slots) any_inflight |= sl->inflight;
            const bool waiting = !S->pending[0].empty() || !S->pending[1].empty() || !S->pending[2].empty();
            if (!any_inflight && waiting) {
                // nothing runs and nothing can be admitted: only more memory would help
                set_error("gbk_server_run_trace: waiting queries cannot be admitted (budget %lld bytes, %lld used)",
                          (long long)S->budget, (long long)S->used());
                return GBK_INSUFFICIENT_SPACE;
            }
            if (!any_inflight && next < nq) {
                const double wait = arrivals[next] - S->now();
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 1e-3)));
            } else {
                std::this_thread::yield();
            }
        }
    }
    for (auto* sl : S->slots) GBK_CUDA(cudaStreamSynchronize(sl->s));
    if (wall_s) *wall_s = S->now();
    for (int64_t i = 0; i < nq; ++i) {
        const QState& q = S->q[i];
        gbk_query_result& r = out[i];
        r.id = i;
        r.kind = q.kind;
        r.source = q.src;
        r.reached = q.dig.reached;
        r.isum = q.dig.isum;
        r.fsum = q.dig.fsum;
        r.iters = q.iters;
        r.batch = q.slot;
        r.t_arrive = q.t_arr;
        r.t_admit = q.t_adm;
        r.t_done = q.t_done;
    }
    return GBK_SUCCESS;
}

int gbk_server_fetch(gbk_server S, int64_t id, void* dst) {
    GBK_REQUIRE(S && dst, GBK_NULL_POINTER, "gbk_server_fetch: NULL argument");
    auto it = S->results.find(id);
    GBK_REQUIRE(it != S->results.end(), GBK_NO_VALUE, "gbk_server_fetch: no kept result for query %lld",
                (long long)id);
    GBK_CUDA(cudaMemcpy(dst, it->second, 4 * (size_t)S->n, cudaMemcpyDeviceToHost));
    return GBK_SUCCESS;
}

int gbk_server_release(gbk_server S, int64_t id) {
    GBK_REQUIRE(S, GBK_NULL_POINTER, "gbk_server_release: NULL argument");
    auto it = S->results.find(id);
    if (it == S->results.end()) return GBK_SUCCESS;
    GBK_CUDA(cudaFree(it->second));
    S->results.erase(it);
    S->result_bytes -= 4 * std::max<int64_t>(S->n, 1);
    return GBK_SUCCESS;
}

int gbk_server_memory(gbk_server S, int64_t* used, int64_t* budget, int32_t* nbatches) {
    GBK_REQUIRE(S, GBK_NULL_POINTER, "gbk_server_memory: NULL argument");
    if (used) *used = S->used();
    if (budget) *budget = S->budget;
    if (nbatches) *nbatches = (int32_t)S->slots.size();
    return GBK_SUCCESS;
}

}  // extern "C"
