/* CPU oracle: a plain-C restatement of the reference algorithms on the
 * SpMV / SpMSpV hot path.  TEST INFRASTRUCTURE ONLY: used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker;
 * never linked into or called by the product library.
 *
 * Each function cites the reference file:line whose behaviour it restates.
 * All graphs are CSR with int32 row pointers and column ids. */
#ifndef GBK_ORACLE_H
#define GBK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Semiring / accumulator / mask vocabulary shared with the checker tests.
 * Values follow include/gbk.h. */
enum { ORC_F32 = 0, ORC_I32 = 1 };

/* y = A x in FP64 from FP32 inputs (spmv.cpp:26-46 check_mxv, in double). */
void orc_spmv_f64(int64_t n, const int32_t* rp, const int32_t* col, const float* val, const float* x,
                  double* y);

/* Generic semiring mxv in the element type, restating
 *   SpMV_all_active_diff_vectors  src/backend/spmv/spmv_csr.h:340-384  (mask == NULL)
 *   SpMV_dense                    src/backend/spmv/spmv_csr.h:266-336  (dense mask)
 * y[i] = accum(y[i], add_j mul(A_ij, x_j)); with a mask, rows outside the
 * mask get y[i] = 0.  `semiring`, `accum` and `mask_mode` take the gbk.h
 * enum values. */
int orc_mxv(int semiring, int accum, int dtype, int64_t n, const int32_t* rp, const int32_t* col,
            const void* val, const void* x, void* y, const void* mask, int mask_dtype, int mask_mode);

/* Push SpMSpV restating src/backend/spmspv/spmspv.h:103-158 and
 * spmspv_atomics.h:5-170: y = identity everywhere, then for every
 * frontier entry (i, x_i) and edge (i -> j): y_j = add(y_j, mul(A_ij, x_i))
 * (or-monoids store 1); with a mask, apply_mask (spmspv.h:17-99). */
int orc_spmspv(int semiring, int accum, int dtype, int64_t n, const int32_t* rp, const int32_t* col,
               const void* val, int64_t nf, const int32_t* f_ids, const void* f_vals, void* y,
               const void* mask, int mask_dtype, int mask_mode);

/* BFS levels: source = 1, unreached = 0, following CSR out-edges
 * (algorithms/bfs/bfs.hpp:93-142, algorithms/bfs/bfs_traditional.hpp:10-48). */
void orc_bfs(int64_t n, const int32_t* rp, const int32_t* col, int32_t source, int32_t* levels);

/* Connected components as the minimum vertex id of each component of the
 * symmetric graph: the fixed point FastSV reaches (algorithms/cc/cc.hpp:12-119). */
void orc_cc(int64_t n, const int32_t* rp, const int32_t* col, int32_t* labels);

/* Single-source shortest paths with integer weights (Dijkstra); unreachable
 * vertices get -1 (algorithms/sssp/sssp_traditional.hpp:8-79,
 * algorithms/sssp/sssp_blast.hpp:8-72). */
void orc_sssp(int64_t n, const int32_t* rp, const int32_t* col, const int32_t* w, int32_t source,
              int64_t* dist);

/* PageRank in FP64 restating algorithms/pr/pr.hpp:20-153 (LAGraph
 * page_rank_sinks with AT = A, d_out = column degree, sinks teleport).
 * Stops after itermax iterations, or earlier once rdiff < tol when tol > 0.
 * Returns the number of iterations run. */
int orc_pagerank(int64_t n, const int32_t* rp, const int32_t* col, double damping, double tol, int itermax,
                 double* rank, double* last_rdiff);

/* Personalised PageRank in FP64 with teleport (and sink mass) to `seed`;
 * same iteration as orc_pagerank otherwise. */
int orc_ppr(int64_t n, const int32_t* rp, const int32_t* col, int32_t seed, double damping, double tol,
            int itermax, double* rank);

/* Triangle count of a symmetric graph: sum(sum((A*A) .* A)) / 6
 * (algorithms/tc/tc.hpp:88-284, Burkhardt). */
uint64_t orc_tc(int64_t n, const int32_t* rp, const int32_t* col);

/* CSR -> CSC transpose (src/backend/matrix/transpose.hpp:68-203); rows
 * ascending within each column. */
void orc_transpose(int64_t n, const int32_t* rp, const int32_t* col, const float* val, int32_t* cp,
                   int32_t* row, float* tval);

/* Graph file reader restating Matrix<T>::init_from_mtx
 * (src/backend/matrix/read_file.hpp:565-617): kind 0 = .mtx text (lines
 * starting with '%' skipped, then "rows cols nnz", then nnz lines of 1-based
 * "row col [value]" read with fgets + sscanf as read_portion does,
 * :5-22; rows keep the file order, as process_portion's push_back gives,
 * :27-47), kind 1 = .mtxbin (int64 rows, cols, nnz, then int64 pairs,
 * :377-400; rows in file order, where the reference's order follows its
 * hash maps).  Blank and '%' lines between entries are skipped.
 * rp == NULL: header only.  Otherwise rp (rows + 1) and col (nnz) are
 * filled.  Returns 0, or 1 = cannot open, 2 = bad header, 3 = malformed
 * line or id out of range (*bad_line = its data-line number, 1-based),
 * 4 = fewer than nnz entries. */
int orc_read_graph_file(const char* path, int kind, int64_t* nrows, int64_t* ncols, int64_t* nnz, int32_t* rp,
                        int32_t* col, int64_t* bad_line);

#ifdef __cplusplus
}
#endif
#endif
