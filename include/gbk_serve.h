/* Query serving over one resident graph: BFS, SSSP and personalised
 * PageRank requests arrive over time and are packed into the batched
 * traversals (gbk_msbfs / gbk_sssp_multi / gbk_ppr lanes) while other
 * queries are running ("continuous batching"): a request takes a free lane
 * as soon as one exists and the device memory it needs fits the server's
 * budget; each batch advances a few iterations per launch on its own CUDA
 * stream, so batches of different kinds overlap on the GPU.
 *
 * The reference answers one query per call (bfs.cpp, sssp.cpp, pr.cpp
 * drivers); the serving loop has no counterpart there.  Results per query
 * equal the single-source algorithms (bfs_blast levels, integer SSSP
 * distances, PPR as gbk_ppr) whether a query runs alone or among others. */
#ifndef GBK_SERVE_H
#define GBK_SERVE_H

#include "gbk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gbk_server_s* gbk_server;

typedef enum gbk_query_kind { GBK_Q_BFS = 0, GBK_Q_PPR = 1, GBK_Q_SSSP = 2 } gbk_query_kind;

typedef struct gbk_server_config {
    int64_t memory_budget;  /* device bytes for batches and kept results; 0 = 80 % of free memory */
    int max_batches[3];     /* per kind (BFS, PPR, SSSP): batches created on demand; 0 = 1 */
    int lanes_per_batch;    /* lanes used per batch: 0 = all (64 BFS, 32 PPR / SSSP); 1 = unbatched */
    int max_inflight;       /* queries running at once over all batches; 0 = no limit, 1 = one at a time */
    int iters_per_launch;   /* iterations between admission points; 0 = 4 */
    int keep_results;       /* 1: keep each result vector on the device until gbk_server_release */
    double ppr_damping;     /* 0 = 0.85 */
    double ppr_tol;         /* 0 = 1e-6 */
    int ppr_itermax;        /* 0 = 100 */
} gbk_server_config;

typedef struct gbk_query_result {
    int64_t id;
    int32_t kind;
    int32_t source;
    int64_t reached;   /* vertices with level > 0 / finite distance / rank > 0 */
    int64_t isum;      /* sum of levels (BFS) or of finite distances (SSSP) */
    double fsum;       /* sum of ranks (PPR) */
    int32_t iters;     /* BFS: largest level; PPR / SSSP: iterations */
    int32_t batch;     /* batch that ran the query */
    double t_arrive;   /* seconds since the trace started */
    double t_admit;
    double t_done;     /* summary available on the host */
} gbk_query_result;

int gbk_server_create(gbk_matrix A, const gbk_server_config* cfg, gbk_server* out);
int gbk_server_destroy(gbk_server s);

/* Replays a request trace in real time: query i of kind kinds[i] from
 * sources[i] arrives arrivals[i] seconds after the start (ascending).  Returns
 * when every query has finished; out[i] receives query i's summary and
 * times, with id = i.  *wall_s (may be NULL) receives the elapsed seconds. */
int gbk_server_run_trace(gbk_server s, const int32_t* kinds, const int32_t* sources, const double* arrivals,
                         int64_t nq, gbk_query_result* out, double* wall_s);

/* With keep_results: copy query id's result vector (n int32 levels, float
 * ranks or int32 distances, INT32_MAX = unreachable) to host memory dst,
 * then (release) free it. */
int gbk_server_fetch(gbk_server s, int64_t id, void* dst);
int gbk_server_release(gbk_server s, int64_t id);

/* Device bytes in use (batches + kept results), the budget, and the number
 * of batches created so far. */
int gbk_server_memory(gbk_server s, int64_t* used, int64_t* budget, int32_t* nbatches);

#ifdef __cplusplus
}
#endif
#endif
