// Batched traversals (internal, not part of the C ABI): many sources or
// right-hand sides advanced together, one lane per query.
//
//  * BFS: 64 lanes packed as the bits of one uint64 per vertex (visited,
//    frontier, next); push (top-down, atomicOr along CSR rows) or pull
//    (bottom-up over CSC rows with early exit) chosen per iteration.
//  * PPR: 32 FP32 columns stored row-interleaved ([n][32]); each iteration is
//    one plus-second SpMM with the teleport / sink / rdiff epilogue fused.
//  * SSSP: 32 int32 distance columns ([n][32]); label-correcting push along
//    CSR rows from the vertices whose distance changed (per-lane bitmasks).
//
// Every batch keeps its state on the device and advances through one CUDA
// graph whose body is a whole iteration and whose `while` node is driven from
// the device (cudaGraphSetConditional in the control kernel): a launch runs
// until no lane is active, until a lane finishes (serving mode) or until a
// per-launch iteration budget is spent.  Lanes are independent: a lane's
// arithmetic never reads another lane's data, so a query's result is the same
// alone or mixed with others.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace gbk {

constexpr int kBfsLanes = 64;
constexpr int kColLanes = 32;

// Host-visible summary of a batch, copied to pinned memory after each launch.
struct BatchStatus {
    unsigned long long active;    // lanes still running
    unsigned long long finished;  // lanes finished and not yet released
    int32_t iter;                 // iterations run by the batch
    int32_t launch_iters;         // iterations run by the last launch
    int32_t iters[64];            // per lane: BFS depth reached, PPR / SSSP iterations
};

enum BatchKind { kBatchBfs = 0, kBatchPpr = 1, kBatchSssp = 2 };

// Per-lane summary of a finished result: vertices reached (BFS level > 0,
// finite distance, rank > 0), the integer sum (levels, distances) and the
// float sum (ranks).
struct LaneDigest {
    long long reached;
    long long isum;
    double fsum;
};

struct Batch {
    virtual ~Batch() {}
    virtual int kind() const = 0;
    virtual int lanes() const = 0;
    // Start queries in the lanes of `mask` (must be idle); src[lane] is the
    // source / seed vertex.  Stream-ordered; no host synchronisation.
    virtual int admit(unsigned long long mask, const int32_t* src, cudaStream_t s) = 0;
    // One graph launch: iterate until no lane is active, or (stop_on_finish)
    // until a lane finishes, or `budget` iterations.  The status is copied to
    // host() on the same stream.
    virtual int launch(int budget, bool stop_on_finish, cudaStream_t s) = 0;
    // The status as of the last launch (valid once the stream passed it).
    virtual const BatchStatus* host() const = 0;
    // Copy the result of finished lanes [lane_lo, lane_lo + nl) to dst,
    // row j = lane lane_lo + j, row stride `stride` elements (levels int32,
    // ranks float, distances int32).
    virtual int extract(int lane_lo, int nl, void* dst, int64_t stride, cudaStream_t s) = 0;
    // Summaries of the finished lanes in `mask` into d_out[lane] (device,
    // lanes() entries; the masked entries are zeroed first).
    virtual int digest(unsigned long long mask, LaneDigest* d_out, cudaStream_t s) = 0;
    // Make finished lanes idle again.
    virtual int release(unsigned long long mask, cudaStream_t s) = 0;
    // Device bytes held by the batch and the bytes of one lane's state.
    virtual size_t device_bytes() const = 0;
    virtual size_t lane_bytes() const = 0;
    // Kernels launched per iteration (for the launch counter).
    virtual int kernels_per_iter() const = 0;
};

int make_bfs_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s);
int make_ppr_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s);
int make_sssp_batch(gbk_matrix A, const BatchOptions& o, Batch** out, cudaStream_t s);

// BFS only: write levels straight into caller memory ([lane][stride]).
int bfs_batch_set_levels(Batch* b, int32_t* levels, int64_t stride, cudaStream_t s);

// The options gbk_batch_autotune chose for this matrix and kind, else the defaults.
BatchOptions base_options(gbk_matrix A, int kind);

}  // namespace gbk
