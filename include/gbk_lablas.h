/* Algorithm entry points of libgbk_lablas.so: the reference's graph
 * algorithms, written against the drop-in lablas:: C++ API
 * (gb_kun_b200/lablas/gb_kun.h) and run on the GPU.  Plain C for callers in
 * other languages (the Python tests and bench bind these with ctypes).
 *
 * A gbk_lablas_graph holds one CSR graph (int32 indices, host arrays copied
 * to the device once) as lablas::Matrix<float> and lablas::Matrix<int>.
 * Every call returns 0 or a gbk_status / LA_Info code; the text of the last
 * failure of the calling thread is in gbk_lablas_get_last_error.  *ms, when
 * not NULL, receives the call's wall time in milliseconds with the device
 * synchronised before and after (graph construction excluded). */
#ifndef GBK_LABLAS_H
#define GBK_LABLAS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gbk_lablas_graph_s* gbk_lablas_graph;

/* weights: NULL for unit weights, else nnz int32 edge weights (SSSP). */
int gbk_lablas_graph_create(gbk_lablas_graph* out, int64_t n, const int32_t* row_ptr, const int32_t* col,
                            const int32_t* weights);
/* Graph from a .mtx / .mtxbin file (or a .gbkcsr CSR cache) through
 * lablas::Matrix<float>::init_from_mtx, as the reference's drivers load a
 * graph file (src/helpers/lib_kernels/init_matrix.h:11-14); unit weights,
 * rows in the file's order.  The file's row and column counts must agree. */
int gbk_lablas_graph_from_file(gbk_lablas_graph* out, const char* path);
int gbk_lablas_graph_destroy(gbk_lablas_graph g);
int gbk_lablas_get_last_error(char* buf, size_t len);

/* bfs_blast (algorithms/bfs/bfs.hpp:94-142): levels, source = 1, unvisited = 0,
 * with the level loop on the device (gbk_bfs_levels). */
int gbk_lablas_bfs(gbk_lablas_graph g, int64_t source, int32_t* levels, double* ms);
/* The same levels through bfs_blast's own sequence of GraphBLAS calls
 * (assign, masked vxm, reduce with a host read per level). */
int gbk_lablas_bfs_ops(gbk_lablas_graph g, int64_t source, int32_t* levels, double* ms);
/* cc (algorithms/cc/cc.hpp:12-119): component labels = smallest vertex id of
 * each component; union-find on the device for a symmetric matrix
 * (*iterations = 0), the FastSV loop otherwise. */
int gbk_lablas_cc(gbk_lablas_graph g, int32_t* labels, int32_t* iterations, double* ms);
/* The FastSV loop as cc.hpp writes it, whatever the matrix
 * (*iterations = its iteration count). */
int gbk_lablas_cc_fastsv(gbk_lablas_graph g, int32_t* labels, int32_t* iterations, double* ms);
/* sssp_bellman_ford_blast (algorithms/sssp/sssp_blast.hpp:8-72) in float
 * (weights as exact floats; unreachable = FLT_MAX). */
int gbk_lablas_sssp_f32(gbk_lablas_graph g, int64_t source, float* dist, double* ms);
/* The same distances through sssp_bellman_ford_blast's own sequence of
 * GraphBLAS calls (vxm, eWiseAdds, masked assign, reduce with a host read per
 * round). */
int gbk_lablas_sssp_f32_ops(gbk_lablas_graph g, int64_t source, float* dist, double* ms);
/* The same rounds in int32 (unreachable = INT32_MAX). */
int gbk_lablas_sssp_i32(gbk_lablas_graph g, int64_t source, int32_t* dist, double* ms);
/* LAGraph page_rank_sinks (algorithms/pr/pr.hpp:20-153); stops after
 * itermax iterations or once rdiff < tol (tol > 0). */
int gbk_lablas_pagerank(gbk_lablas_graph g, int32_t itermax, double damping, double tol, float* ranks,
                        int32_t* iterations, double* ms);
/* The same iteration as page_rank_sinks' own sequence of GraphBLAS calls
 * (a host read of rdiff per iteration). */
int gbk_lablas_pagerank_ops(gbk_lablas_graph g, int32_t itermax, double damping, double tol, float* ranks,
                        int32_t* iterations, double* ms);
/* Personalised PageRank from one seed through the same lablas:: steps
 * (one plus-second mxv per iteration); teleport and sink mass return to the
 * seed.  The single-query path the batched gbk_ppr is compared with. */
int gbk_lablas_ppr(gbk_lablas_graph g, int64_t seed, int32_t itermax, double damping, double tol, float* ranks,
                   int32_t* iterations, double* ms);
/* Burkhardt triangle count (algorithms/tc/tc.hpp:209-217); the graph must be symmetric. */
int gbk_lablas_tc(gbk_lablas_graph g, uint64_t* count, double* ms);
/* LAGr_TriangleCount with a method (algorithms/tc/tc.hpp:17-26): 0 default,
 * 1 Burkhardt, 2 Cohen, 3 Sandia, 4 Sandia2, 5 SandiaDot, 6 SandiaDot2;
 * presort NoSort.  The reference's L / U keep A's structure, so every method
 * returns its Burkhardt count. */
int gbk_lablas_tc_method(gbk_lablas_graph g, int32_t method, uint64_t* count, double* ms);
/* y = A x through lablas::mxv (plus-times, f32) in the given storage format
 * (MatrixStorageFormat value: 0 CSR, 3 CSR_SEG, 4 LAV, 6 SELL_C); vals are
 * the nnz matrix values. */
int gbk_lablas_spmv(gbk_lablas_graph g, int32_t format, const float* vals, const float* x, float* y, double* ms);

#ifdef __cplusplus
}
#endif
#endif
