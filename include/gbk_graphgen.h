/* Seeded synthetic graph inputs (host library libgbk_graphgen.so).
 *
 * Replaces the reference's time-seeded generators:
 *   GraphGenerationAPI::RMAT            src/helpers/graph_generation/graph_generation.hpp:93-191
 *   GraphGenerationAPI::random_uniform  src/helpers/graph_generation/graph_generation.hpp:37-89
 *   EdgeListContainer::remove_duplicated_edges  src/helpers/graph_generation/edges_container.hpp:32-152
 *   select_non_trivial_vertex           src/helpers/lib_kernels/select_non_vertex.hpp:5-24
 * Every draw is a pure function of (seed, counter): identical output on any
 * host and thread count.  Graphs are de-duplicated and free of self loops;
 * CSR columns are sorted ascending within each row. */
#ifndef GBK_GRAPHGEN_H
#define GBK_GRAPHGEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { GBK_GEN_OK = 0, GBK_GEN_BAD_ARG = 1, GBK_GEN_NO_MEMORY = 2, GBK_GEN_TOO_LARGE = 3 };

typedef struct gbk_graph {
    int64_t n;        /* vertices (rows == cols) */
    int64_t nnz;      /* directed edges after de-duplication */
    int32_t* row_ptr; /* n + 1 */
    int32_t* col;     /* nnz, ascending within a row */
} gbk_graph;

/* R-MAT with 2^scale vertices and edge_factor * 2^scale generated edges
 * (quadrant probabilities a, b, c; d = 1 - a - b - c).  Reference drivers
 * pass 57/19/19/5 (src/helpers/lib_kernels/init_matrix.h:32). */
int gbk_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int undirected,
                 gbk_graph** out);
/* Erdos-Renyi G(n, m): m = edge_factor * 2^scale uniform edges. */
int gbk_gen_uniform(int scale, int edge_factor, uint64_t seed, int undirected, gbk_graph** out);
/* Explicit edge list -> de-duplicated CSR (used for small fixtures). */
int gbk_gen_from_edges(int64_t n, int64_t m, const int64_t* src, const int64_t* dst, int undirected,
                       gbk_graph** out);
void gbk_graph_free(gbk_graph* g);

/* Edge values uniform in [0,1) (24-bit), symmetric in (i, j). */
void gbk_gen_values_f32(int64_t n, const int32_t* row_ptr, const int32_t* col, uint64_t seed, float* out);
/* Integer edge weights uniform in [lo, hi], symmetric in (i, j). */
void gbk_gen_weights_i32(int64_t n, const int32_t* row_ptr, const int32_t* col, uint64_t seed, int32_t lo,
                         int32_t hi, int32_t* out);
/* Dense vector uniform in [0,1) (24-bit). */
void gbk_gen_vector_f32(int64_t n, uint64_t seed, float* out);
/* `count` seeded vertices with non-zero out-degree; returns how many were found. */
int64_t gbk_gen_sources(int64_t n, const int32_t* row_ptr, int64_t count, uint64_t seed, int32_t* out);

/* Graph files for ingest tests and benchmarks, entries in the given order.
 * .mtx: Matrix Market coordinate text, 1-based, "pattern" or (vals != NULL)
 * "real" with a %g value column.  .mtxbin: int64 rows, cols, nnz, then int64
 * 1-based (src, dst) pairs, the layout binary_read_mtx_file reads
 * (src/backend/matrix/read_file.hpp:377-400). */
int gbk_gen_write_mtx(const char* path, int64_t nrows, int64_t ncols, int64_t nnz, const int32_t* src,
                      const int32_t* dst, const float* vals);
int gbk_gen_write_mtxbin(const char* path, int64_t nrows, int64_t ncols, int64_t nnz, const int32_t* src,
                         const int32_t* dst);

#ifdef __cplusplus
}
#endif
#endif
