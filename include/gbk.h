/* gbk: C ABI of the B200 GraphBLAS hot path (libgbk.so).
 *
 * This is the boundary beneath the reference's backend:: layer
 * (src/backend/operations/operations.h).  Every entry point takes plain
 * pointers and sizes and returns a gbk_status; no entry point throws.
 * Vectors are device arrays owned by the caller; matrices are opaque
 * handles that own their device storage (CSR, CSC and the optional
 * optimised format for both orientations, as backend::Matrix owns
 * csr_data / csc_data / data / transposed_data, src/backend/matrix/matrix.h:179-188).
 *
 * Streams: every launch goes to the `stream` argument (a cudaStream_t,
 * NULL = legacy default stream).  Calls that share a matrix must be ordered
 * on one stream (the matrix holds per-call scratch), unless stated otherwise.
 */
#ifndef GBK_H
#define GBK_H

#include <stddef.h>
#include <stdint.h>

#include "gbk_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gbk_matrix_s* gbk_matrix;

/* Optional storage-format parameters (gbk_matrix_set_format). Zero fields
 * take the defaults stated per field. */
typedef struct gbk_format_params {
    int32_t sell_c;          /* SELL-C slice height; default 32 (one slice per warp) */
    int32_t sell_sigma;      /* SELL-C sorting window in rows; default 4096; 1 = no sort */
    int32_t seg_cols;        /* CSR_SEG / LAV column-segment width; default 131072 (512 KiB of f32 x) */
    float lav_dense_frac;    /* LAV: fraction of nnz in the dense column segments; default 0.8 */
    int32_t csr_kernel;      /* CSR kernel: 0 default (degree bins; unmasked products over matrices of
                                2^23 or more entries use kernel 3), 1 merge-path tiles, 2 degree bins,
                                3 equal runs of 256 entries per warp (needs 16-byte aligned column / value
                                arrays, which the library's own allocations always are; otherwise, and
                                for semirings whose add is not associative, the degree bins or the
                                in-order row kernel run) */
    int32_t sell_hot_cols;   /* SELL-C: columns renumbered by in-degree and the x values of the first
                                sell_hot_cols (most used) columns staged in shared memory per CTA;
                                0 = off; at most 53248 */
    int32_t sell_reorder_cols; /* SELL-C: renumber columns by in-degree (most used first) so gathers of
                                  popular x values share sectors and L1 lines; implied by sell_hot_cols */
    int32_t seg_staged;      /* CSR_SEG / LAV: 0 (default) windows of 49152 columns whose x values are
                                staged in shared memory, row sums folded into y atomically; -1 =
                                seg_cols-wide segments gathered from L2 and merged per row in segment
                                order.  SELL-C: 1 = SELL-C-sigma built inside staged windows of 45056
                                columns (sigma = the window, virtual rows in pieces of at most 32 entries;
                                sell_reorder_cols renumbers the columns by in-degree first); 0 (default)
                                = the gathered SELL-C */
} gbk_format_params;

/* A mask argument: either dense (n entries of `dtype`, non-zero = set) or
 * sparse (`nvals` ascending vertex ids), the two forms backend::Vector
 * switches between (src/backend/vector/vector.h:81-129). */
typedef struct gbk_mask {
    const void* dense;    /* NULL when the mask is sparse */
    int32_t dtype;        /* gbk_dtype of `dense` */
    int32_t mode;         /* gbk_mask_mode */
    const int32_t* ids;   /* sparse form; used when dense == NULL */
    int64_t nvals;
} gbk_mask;

typedef struct gbk_matrix_info {
    int64_t nrows, ncols, nnz;
    int32_t vtype;           /* gbk_dtype */
    int32_t format;          /* gbk_format */
    int64_t padded_nnz;      /* stored entries of the optimised format (A orientation) */
    int64_t device_bytes;    /* all device storage owned by the handle */
    int64_t ntiles;          /* merge-path tiles of the CSR orientation */
    int32_t has_csc;
} gbk_matrix_info;

/* ---- library ------------------------------------------------------------ */

/* Select the device and check it is an sm_100 part. */
int gbk_init(int device);
/* Copy the last error text of the calling thread into buf (NUL-terminated). */
int gbk_get_last_error(char* buf, size_t len);
/* Number of kernel launches issued by this library since load (all threads). */
int64_t gbk_launch_count(void);

/* ---- matrices ----------------------------------------------------------- */

/* Create a matrix from CSR arrays (int32 row pointers and column ids).
 * on_device = 0: the arrays are host memory and are copied; 1: device
 * memory, copied device-to-device.  Replaces lablas::Matrix<T>::
 * build_from_csr_arrays (src/cpp_graphblas/matrix.hpp:93-105 ->
 * src/backend/matrix/build.hpp:170-210).  The CSC (A^T) is built on the
 * device on first use. */
int gbk_matrix_create_csr(gbk_matrix* out, int64_t nrows, int64_t ncols, int64_t nnz, const int32_t* row_ptr,
                          const int32_t* col, const void* val, gbk_dtype vtype, int on_device, void* stream);
int gbk_matrix_destroy(gbk_matrix A);
int gbk_matrix_get_info(gbk_matrix A, gbk_matrix_info* info);
/* Device pointers of the CSR (transpose = 0) or CSC (transpose = 1) arrays. */
int gbk_matrix_csr_arrays(gbk_matrix A, int transpose, const int32_t** ptr, const int32_t** idx,
                          const void** val, void* stream);
/* Build the optimised storage format for A and A^T, replacing
 * Matrix<T>::init_optimized_structures (src/backend/matrix/build.hpp:5-118).
 * GBK_FMT_CSR drops any optimised format. */
int gbk_matrix_set_format(gbk_matrix A, gbk_format fmt, const gbk_format_params* params, void* stream);

typedef struct gbk_tune_result {
    int32_t format;          /* chosen gbk_format */
    int32_t sell_sigma;      /* chosen SELL-C window (SELL-C only) */
    int32_t csr_kernel;      /* chosen CSR kernel (CSR only) */
    int32_t cached;          /* 1 when the choice came from the cache (nothing was timed) */
    int32_t ncandidates;
    float best_ms;
    float candidate_ms[16];  /* CSR bins, CSR merge-path, SELL-C sigma 1 / 256 / 4096, CSR_SEG, LAV,
                                SELL-C sigma 4096 with 16384 / 53248 hot columns, sigma 256 with 53248,
                                SELL-C sigma 4096 / 256 with renumbered columns, SELL-C in staged x
                                windows without / with renumbered columns, CSR in runs of 256 entries
                                per warp; unused entries 0 */
    int32_t sell_hot_cols;   /* chosen hot-column count (SELL-C only; -1 = renumbered columns) */
    int32_t sell_staged;     /* 1 when the chosen SELL-C runs inside staged x windows */
} gbk_tune_result;

/* Per-graph autotuner (no counterpart in the reference, which takes the
 * format from its -format flag, src/helpers/cmd_parser/cmd_parser.hpp, and
 * fixes C / sigma at compile time, src/backend/la_backend.h:16-34): times
 * `reps` unmasked SpMVs of every candidate format / kernel for the given
 * orientation and semiring, keeps the fastest on A, and caches the choice by
 * graph fingerprint (process-wide, plus the file GBK_TUNE_CACHE if set). */
int gbk_matrix_autotune(gbk_matrix A, int transpose, gbk_semiring sr, int32_t reps, gbk_tune_result* result,
                        void* stream);

/* ---- SpMV / SpMSpV ------------------------------------------------------ */

/* y = accum(y, A (+.x) x) over a semiring, every operand of type `dtype`
 * (GBK_F32 or GBK_I32).  transpose = 0 is mxv (rows of A, backend::SpMV,
 * src/backend/spmv/spmv.h:20-79); transpose = 1 is vxm (rows of A^T,
 * backend::VSpM, spmv.h:83-146).  mask: NULL or a dense array of n
 * mask_dtype entries; rows the mask selects (mask_mode GBK_MASK_STR_COMP
 * complements, every other mode does not) get accum(y, result), other rows
 * get 0 (SpMV_dense, src/backend/spmv/spmv_csr.h:266-336).  Unmasked calls
 * use the optimised format chosen by gbk_matrix_set_format.  x may alias y. */
int gbk_mxv(gbk_matrix A, int transpose, gbk_semiring sr, gbk_binop accum, gbk_dtype dtype, const void* x,
            void* y, const void* mask, gbk_dtype mask_dtype, gbk_mask_mode mask_mode, void* stream);

/* gbk_mxv with a sparse mask: rows listed in mask_ids get accum(y, result)
 * and other rows keep y, unless mask_mode is GBK_MASK_STR_COMP, where listed
 * rows get 0 and the others accum(y, result) (SpMV_sparse,
 * src/backend/spmv/spmv_csr.h:175-262). */
int gbk_mxv_sparse_mask(gbk_matrix A, int transpose, gbk_semiring sr, gbk_binop accum, gbk_dtype dtype,
                        const void* x, void* y, const int32_t* mask_ids, int64_t mask_nvals, gbk_mask_mode mask_mode,
                        void* stream);

/* Push SpMSpV: y = identity, then for every frontier entry (i, x_i) and
 * every stored A(r, i) (transpose = 0, mxv: the CSC column i) or A(i, r)
 * (transpose = 1, vxm: the CSR row i): y_r = add(y_r, mul(A, x_i)).  The
 * update is chosen as the reference does by probing add(3, 5): 8 -> atomic
 * add, 1 -> store 1, else an atomic read-modify-write with add
 * (src/backend/spmspv/spmspv.h:103-158, spmspv_atomics.h:5-170).  With a
 * mask, apply_mask follows (spmspv.h:17-99): selected rows get
 * accum(old y, y), other rows 0 (a sparse mask without complement leaves
 * unlisted rows as computed).  Without a mask the accumulator is not used. */
int gbk_spmspv(gbk_matrix A, int transpose, gbk_semiring sr, gbk_binop accum, gbk_dtype dtype,
               const int32_t* x_ids, const void* x_vals, int64_t x_nvals, void* y, const gbk_mask* mask,
               void* stream);
/* Push SpMSpV with a sparse output (spmspv_unmasked_or_map /
 * spmspv_unmasked_critical_map, src/backend/spmspv/spmspv_maps.h:5-142, the
 * SparseVector form of backend::SpMSpV, spmspv.h:162-205): every row reached
 * from the frontier appears once in (y_ids, y_vals), ids ascending, its value
 * the semiring's add over its products; when add probes to 1 (or-monoids)
 * every reached row holds 1.  y_ids / y_vals need room for the number of rows
 * of the output (at most the distinct reached rows are written); *y_nvals is
 * written on the host (the call synchronises the stream).  A mask is refused
 * (GBK_UNSUPPORTED) as the reference throws for it. */
int gbk_spmspv_sparse(gbk_matrix A, int transpose, gbk_semiring sr, gbk_dtype dtype, const int32_t* x_ids,
                      const void* x_vals, int64_t x_nvals, int32_t* y_ids, void* y_vals, int64_t* y_nvals,
                      const gbk_mask* mask, void* stream);

/* ---- SpGEMM ------------------------------------------------------------- */

/* Masked SpGEMM C<M> = A (+.x) B: C gets the structure of M and, at every
 * stored (i, j) of M, the semiring sum over k in row i of A and column j
 * of B (GBK_PLUS_ONE counts common k, GBK_PLUS_TIMES sums products).
 * Replaces SpMSpM_masked_ikj (src/backend/spmspm/spmspm_masked_hash_based_gustavson.h:9-168)
 * as used by Burkhardt triangle counting (algorithms/tc/tc.hpp:209-217).
 * Rows of A must be column-sorted (lablas::Matrix keeps them so); B's
 * columns are read from its device CSC.  *out is a new matrix of ctype
 * (GBK_I32 or GBK_F32) values. */
int gbk_mxm_masked(gbk_matrix* out, gbk_matrix M, gbk_matrix A, gbk_matrix B, gbk_semiring sr, gbk_dtype ctype,
                   void* stream);

/* Unmasked SpGEMM C = A (+.x) B, replacing SpMSpM_unmasked_ikj
 * (src/backend/spmspm/spmspm_hash_based_gustavson.h:9-148, reached by mxm
 * with a NULL mask, src/backend/operations/operations.h:476-482): every
 * product A_ik * B_kj is added into C_ij with the semiring's add and entries
 * whose sum is 0 are dropped (the reference keeps val != 0).  A and B share
 * a value type (GBK_F32 / GBK_I32), which C takes; rows of C are
 * column-sorted (the reference's order follows its hash maps).  Semirings:
 * plus-times, plus-second, plus-one, min-plus, min-second, or-and. */
int gbk_mxm(gbk_matrix* out, gbk_matrix A, gbk_matrix B, gbk_semiring sr, void* stream);

/* Triangle count with Burkhardt's result, sum (sum ((A * A) .* A)) / 6
 * (algorithms/tc/tc.hpp:209-217).  For a symmetric A without self loops
 * (checked on the device against its CSC) each edge is oriented from its
 * (degree, id)-smaller end and every triangle counted once by intersecting
 * the oriented neighbour lists, which gives the same number; any other A
 * takes the masked plus-one product as the formula stands. */
int gbk_triangle_count(gbk_matrix A, uint64_t* count, void* stream);

/* ---- select ---------------------------------------------------------------- */

/* Index-unary operators of select: index ops keep a_ij by position (k = the
 * thunk), value ops by comparing a_ij with the thunk. */
typedef enum gbk_select_op {
    GBK_SEL_TRIL = 0,      /* j <= i + k */
    GBK_SEL_TRIU = 1,      /* j >= i + k */
    GBK_SEL_DIAG = 2,      /* j == i + k */
    GBK_SEL_OFFDIAG = 3,   /* j != i + k */
    GBK_SEL_VALUE_EQ = 4,
    GBK_SEL_VALUE_NE = 5,
    GBK_SEL_VALUE_GT = 6,
    GBK_SEL_VALUE_GE = 7,
    GBK_SEL_VALUE_LT = 8,
    GBK_SEL_VALUE_LE = 9
} gbk_select_op;

/* Matrix select as backend::select (src/backend/operations/select.h:363-395):
 * the result keeps every stored entry of A (the structure does not change);
 * an entry's value is a_ij where the operator keeps it and 0 where not. */
int gbk_select_matrix(gbk_matrix* out, gbk_matrix A, gbk_select_op op, double thunk, void* stream);
/* Vector select (select.h:17-315): for every i the mask selects (all i with
 * mask == NULL; a dense mask selects non-zero entries, a sparse one its ids,
 * COMP / SCMP / STR_COMP complement), w[i] = accum(w[i], r) with r = u[i]
 * if the operator keeps (u[i], i, 0) and 0 if not; unselected i get 0 when
 * replace != 0 (GrB_REPLACE) and keep w[i] otherwise. */
int gbk_select_vector(gbk_select_op op, double thunk, void* w, gbk_dtype wt, const void* u, gbk_dtype ut,
                      int64_t n, gbk_binop accum, const gbk_mask* mask, int replace, void* stream);

/* ---- batched traversals (many sources per launch) ----------------------- */

/* Multi-source BFS: up to 64 sources advanced together, one bit of a uint64
 * per vertex each.  Per source the result equals bfs_blast
 * (algorithms/bfs/bfs.hpp:93-142, edges followed along the rows of A):
 * levels[k * n + v] = depth of v from sources[k] (source 1, unreached 0).
 * levels is device memory of nsources * n int32.  direction: 0 chooses push
 * or pull per iteration, 1 push only, 2 pull only (same levels).  depths
 * (host, may be NULL) receives each source's largest level.  The whole
 * iteration loop runs as one CUDA graph; synchronises the stream.  The
 * reference runs one source per call; the packing is this library's. */
int gbk_msbfs(gbk_matrix A, const int32_t* sources, int nsources, int32_t* levels, int direction, int32_t* depths,
              void* stream);
/* Personalised PageRank for up to 32 seeds as one FP32 SpMM per iteration.
 * Per seed it is the page_rank_sinks iteration (algorithms/pr/pr.hpp:20-153)
 * with r0 = e_seed and the teleport and sink mass returned to the seed:
 * r = [(1 - damping) + damping * sink] e_seed + A (r ./ d), d = max(coldeg,
 * 1) / damping, stopping when sum |r_new - r| < tol (tol > 0) or after
 * itermax iterations.  ranks is device memory of nseeds * n floats (row k =
 * seed k); iters (host, may be NULL) receives the iterations per seed.
 * Synchronises the stream. */
int gbk_ppr(gbk_matrix A, const int32_t* seeds, int nseeds, double damping, double tol, int itermax, float* ranks,
            int32_t* iters, void* stream);
/* Single-source shortest paths from up to 32 sources with integer edge
 * weights (the matrix values; GBK_F32 values are truncated to int32).
 * dist[k * n + v] = shortest distance from sources[k] (INT32_MAX when
 * unreachable), the fixpoint sssp_bellman_ford_blast reaches
 * (algorithms/sssp/sssp_blast.hpp:8-72).  iters (host, may be NULL) receives
 * the relaxation rounds per source.  Weights must be non-negative.
 * Synchronises the stream. */
int gbk_sssp_multi(gbk_matrix A, const int32_t* sources, int nsources, int32_t* dist, int32_t* iters, void* stream);

/* ---- single-query traversals (the whole loop on the device) ------------- */

/* Single-source BFS with the result of bfs_blast (algorithms/bfs/bfs.hpp:94-142,
 * edges followed along the rows of A): levels[v] = 1 for the source, k + 1 at
 * distance k, 0 unreached.  levels is device memory of n elements of
 * level_type (GBK_F32 as the reference's Vector<float>, GBK_I32, GBK_I64,
 * GBK_F64).  Direction-optimising: each level expands top-down from a queue
 * or bottom-up over the unvisited vertices' in-edges (the CSC, built on first
 * use) as the frontier's edge count decides (direction 0; 1 top-down only,
 * 2 bottom-up only, same levels); the level loop runs as one CUDA graph with
 * a device-side `while` node, so the call issues one graph launch whatever
 * the depth.  depth (host, may be NULL) receives the largest level and then
 * the call synchronises the stream; with depth NULL it does not. */
int gbk_bfs_levels(gbk_matrix A, int64_t source, int direction, gbk_dtype level_type, void* levels, int32_t* depth,
                   void* stream);
/* Single-source shortest paths with the distances of sssp_bellman_ford_blast
 * (algorithms/sssp/sssp_blast.hpp:8-72): dist[v] = the smallest sum of edge
 * values (the matrix values) over the walks from source to v, added left to
 * right in the matrix's value type (GBK_F32: float, FLT_MAX = unreachable;
 * GBK_I32: saturating int32, INT32_MAX = unreachable); dist[source] = 0.
 * dist is device memory of n elements of the matrix's value type.  A
 * label-correcting near-far worklist: each round relaxes the out-edges (rows
 * of A) of the vertices whose distance dropped below a threshold; vertices at
 * or above it wait in a far pile until the threshold rises by delta.  delta
 * 0 picks 8 x the mean edge value / the mean row length (sampled), delta < 0
 * turns the pile off (plain worklist); the distances are the same either way.
 * All rounds run as one CUDA graph with a device-side `while` node.  Negative
 * edge values are allowed; with a negative cycle reachable the rounds stop
 * after 2n + 1 and the distances are not defined (the reference's n-round
 * bound gives other values there).  rounds (host, may be NULL) receives the
 * rounds run and then the call synchronises the stream; with rounds NULL and
 * delta != 0 it does not. */
int gbk_sssp_dist(gbk_matrix A, int64_t source, double delta, void* dist, int32_t* rounds, void* stream);
/* PageRank as page_rank_sinks (algorithms/pr/pr.hpp:20-153) on the graph
 * whose edge j -> i is the entry a_ij (the reference's AT): r0 = 1/n; each
 * iteration r = teleport + A (r_old ./ d) with d = max(coldeg / damping,
 * 1 / damping) in float (coldeg = entries in the column), teleport =
 * (1 - damping) / n + damping / n * sink, where sink is the reference's sink
 * mass: the sum of r_old over the columns without entries when there are
 * more than 0.3 n of them, and otherwise the sum of r_old[0 .. nsinks - 1]
 * (its sparse sink vector is read at list positions, not at vertex ids:
 * src/backend/operations/generic_operations.h:28-34 with operations.h:63-65).
 * The loop stops after itermax iterations, or earlier once
 * sum |r_old - r| < tol when tol > 0.  A's values must be GBK_F32 (they are
 * not read: plus-second).  ranks is device memory of n floats.  The SpMV runs
 * in A's storage format (gbk_matrix_set_format / gbk_matrix_autotune); after
 * the first iteration the loop runs as one CUDA graph.  The element-wise
 * sums are formed in a fixed order, so with the CSR format a run repeats bit
 * for bit; the staged formats fold row pieces with atomics, whose order can
 * move the last bits between runs.  iters and rdiff
 * (host, may be NULL) receive the iterations run and the last sum
 * |r_old - r|.  Synchronises the stream. */
int gbk_pagerank(gbk_matrix A, int32_t itermax, double damping, double tol, float* ranks, int32_t* iters,
                 float* rdiff, void* stream);
/* *symmetric = 1 when A is square and its pattern equals its transpose's with
 * every row's column indices ascending, else 0 (an unsorted symmetric matrix
 * reads as 0).  Computed once per matrix on the device against its CSC. */
int gbk_matrix_pattern_symmetric(gbk_matrix A, int32_t* symmetric, void* stream);
/* Connected components as the label of each vertex = the smallest vertex id
 * of its component: the fixed point of the FastSV loop in cc
 * (algorithms/cc/cc.hpp:12-119) on a symmetric A.  Lock-free union-find over
 * the stored edges, each linking the larger root under the smaller, then one
 * pass taking every vertex's root: three kernel launches, no host round
 * trip.  Edges count in both directions, so a non-symmetric A gets its weakly
 * connected components (FastSV's answer can differ there; callers that must
 * reproduce it check gbk_matrix_pattern_symmetric first).  labels is device
 * memory of n elements of label_type (GBK_I32, GBK_I64 or GBK_F32). */
int gbk_cc_labels(gbk_matrix A, gbk_dtype label_type, void* labels, void* stream);

/* Tuning of the batched traversals on this graph: times each candidate on
 * the given sources (CUDA events, best of 2 after a warm-up) and keeps the
 * fastest for later gbk_msbfs / gbk_ppr / gbk_sssp_multi calls and servers
 * on A.  kind: 0 BFS (candidates: push/pull switch factor 2, 4, 8, 14, push
 * only, pull only), 1 PPR and 2 SSSP (edges per work item 64 .. 1024).  The
 * reference has no tuner; it takes its format from the command line. */
typedef struct gbk_batch_tune_result {
    int32_t kind;
    int32_t item_edges;     /* chosen edges per work item (PPR / SSSP) */
    int32_t bfs_direction;  /* chosen BFS direction mode */
    int32_t bfs_alpha;      /* chosen push -> pull switch factor */
    int32_t ncandidates;
    float best_ms;
    float candidate_ms[8];
} gbk_batch_tune_result;
int gbk_batch_autotune(gbk_matrix A, int kind, const int32_t* sources, int nsources, gbk_batch_tune_result* out,
                       void* stream);

/* ---- vectors ------------------------------------------------------------ */

/* Count of non-zero entries (DenseVector::get_nvals, dense_vector.hpp:44-52).
 * Writes *out on the host; synchronises the stream. */
int gbk_vec_nvals(const void* v, gbk_dtype t, int64_t n, int64_t* out, void* stream);
/* Dense -> sparse: ids ascending and their values (SparseVector::convert,
 * sparse_vector.hpp:35-92).  ids / vals need room for n entries.  Writes
 * *nvals on the host; synchronises the stream. */
int gbk_vec_to_sparse(const void* dense, gbk_dtype t, int64_t n, int32_t* ids, void* vals, int64_t* nvals,
                      void* stream);
/* The same conversion without allocating device memory (no counterpart in
 * the reference).  For callers that cannot allocate at call time: a host
 * framework whose caching allocator already holds the free device memory,
 * a serving loop that must not wait on the allocator mid-request, an
 * application that budgets device memory up front.  Its scratch is a fixed
 * ~32 KiB array inside the library, held on every GPU that loads it until
 * exit, so n is limited to 33,554,432 (larger n: GBK_INVALID_VALUE).  All
 * calls share the scratch: calls that overlap on the GPU race.  gbk_init
 * loads this entry point's code and scratch on its device and caches the
 * scratch address, so the calls themselves allocate nothing; on a device
 * that never saw gbk_init the first call does that set-up (which may
 * allocate).  After cudaDeviceReset call gbk_init again.  Synchronises the
 * stream (it reads the count back), so it cannot be captured into a CUDA
 * graph. */
int gbk_vec_to_sparse_noalloc(const void* dense, gbk_dtype t, int64_t n, int32_t* ids, void* vals,
                              int64_t* nvals, void* stream);
/* Sparse -> dense: zero fill, then scatter (DenseVector::convert, dense_vector.hpp:87-102). */
int gbk_vec_to_dense(const int32_t* ids, const void* vals, int64_t nvals, gbk_dtype t, void* dense, int64_t n,
                     void* stream);
/* v[i] = value (set_all_constant); value is exact for int32 and float. */
int gbk_vec_fill(void* v, gbk_dtype t, int64_t n, double value, void* stream);
/* v[i] = i (fillAscending). */
int gbk_vec_iota(void* v, gbk_dtype t, int64_t n, void* stream);
/* dst[i] = (dt) src[i]. */
int gbk_vec_cast(const void* src, gbk_dtype st, void* dst, gbk_dtype dt, int64_t n, void* stream);

/* w[i] = op(u[i], v[i]) computed in optype, for every i the mask selects
 * (eWiseAdd / eWiseMult, operations.h:216-267 via generic_dense_vector_op,
 * generic_operations.h:119-164: dense masks select non-zero entries,
 * sparse masks their ids; the mask mode is not consulted).  mask may be NULL. */
int gbk_ewise(gbk_binop op, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut, const void* v,
              gbk_dtype vt, int64_t n, const gbk_mask* mask, void* stream);
/* apply (operations.h:272-341): kind 0 w = unop(u) (op is a gbk_unop);
 * kind 1 w = op(scalar, u); kind 2 w = op(u, scalar) (op is a gbk_binop). */
int gbk_apply(int kind, int op, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut,
              double scalar, int64_t n, const gbk_mask* mask, void* stream);
/* Scalar assign (operations.h:15-45, 80-112 via generic_dense_vector_op_assign,
 * generic_operations.h:11-65 and indexed_dense_vector_op_assign,
 * indexed_operations.h:12-47): w[i] = value for each selected i; a dense
 * mask selects non-zero entries under DEFAULT / STRUCTURE and zero entries
 * under STR_COMP, and nothing under COMP / SCMP.  With indices (device
 * array of nindices entries of index_t), w[idx[k]] = value (a mask, if
 * any, must then be dense and is tested at idx[k]). */
int gbk_assign_scalar(void* w, gbk_dtype wt, int64_t n, double value, const gbk_mask* mask, const void* indices,
                      gbk_dtype index_t, int64_t nindices, void* stream);
/* Vector assign (operations.h:50-77, 115-147) and assignScatter: w[i] =
 * accum(w[i], u[j]) with j = i, except for a sparse DEFAULT / STRUCTURE
 * mask, where i = ids[k] and j = k (the reference reads u at the mask-list
 * position, generic_operations.h:28-34).  With indices: w[idx[k]] =
 * accum(w[idx[k]], u[k]); a repeated index takes the largest k, the result
 * of the sequential order. */
int gbk_assign_vector(gbk_binop accum, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut,
                      int64_t n, const gbk_mask* mask, const void* indices, gbk_dtype index_t, int64_t nindices,
                      void* stream);
/* extract (operations.h:401-430): with indices, w[i] = accum(w[i], u[idx[i]])
 * for i < nindices (a dense mask, if any, tested at idx[i]); without,
 * w[i] = accum(w[i], u[i]) where a dense mask is non-zero, or
 * w[k] = accum(w[k], u[ids[k]]) for a sparse mask (generic_operations.h:68-113). */
int gbk_extract(gbk_binop accum, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut, int64_t n,
                const gbk_mask* mask, const void* indices, gbk_dtype index_t, int64_t nindices, void* stream);
/* *result (host, of type rt) = monoid fold of u's n entries, starting from
 * the monoid identity (operations.h:346-378).  Float sums accumulate in
 * double.  Synchronises the stream. */
int gbk_reduce(gbk_monoid monoid, gbk_dtype rt, const void* u, gbk_dtype ut, int64_t n, void* result,
               void* stream);

#ifdef __cplusplus
}
#endif
#endif
