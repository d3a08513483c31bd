/* Graph ingest for the gbk C ABI: graph files -> device CSR, and a binary CSR
 * cache for fast reloads.
 *
 * Replaces the reference's graph-file path, lablas::Matrix<T>::init_from_mtx
 * (src/cpp_graphblas/matrix.hpp:107-110) -> backend::Matrix<T>::init_from_mtx
 * (src/backend/matrix/read_file.hpp:565-617) with its readers
 * read_mtx_file_pipelined (read_file.hpp:52-165) and binary_read_mtx_file
 * (read_file.hpp:377-561).  The reference has no CSR cache.
 *
 * All functions return a gbk status (0 = success; codes as in gbk.h).
 */
#ifndef GBK_INGEST_H
#define GBK_INGEST_H

#include <stddef.h>
#include <stdint.h>

#include "gbk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gbk_file_kind {
    GBK_FILE_MTX = 0,     /* Matrix Market coordinate text, 1-based "row col [value]" lines */
    GBK_FILE_MTXBIN = 1,  /* the reference's binary edge list: int64 rows, cols, nnz, then nnz int64 pairs */
    GBK_FILE_CSR = 2      /* this library's CSR cache (gbk_matrix_save_csr) */
} gbk_file_kind;

typedef struct gbk_file_info {
    int64_t nrows, ncols, nnz;  /* from the file's header */
    int64_t file_bytes;
    int64_t data_offset;        /* first byte after the header */
    int32_t kind;               /* gbk_file_kind, from the file name's ending */
    int32_t vtype;              /* CSR cache: the stored gbk_dtype; otherwise -1 */
} gbk_file_info;

/* Header of a graph file: .mtx (lines starting with '%' skipped, then
 * "rows cols nnz", read_file.hpp:64-76), .mtxbin (three int64,
 * read_file.hpp:207-213) or a CSR cache (.gbkcsr). */
int gbk_file_info_read(const char* path, gbk_file_info* info);

/* Matrix from a graph file, parsed on the device.  As
 * Matrix<T>::init_from_mtx: 1-based ids, every entry gets the value 1
 * (EDGE_VAL, src/helpers/graph_generation/graph_generation.hpp:6),
 * duplicates are kept, a .mtx value column is ignored and only the first
 * nnz entry lines are read.  Entries of a row keep the file's order (the
 * reference's .mtx path does the same; its .mtxbin path orders a row by
 * hash-map iteration, read_file.hpp:428-476, which is not reproducible).
 * Unlike the reference, which crashes or reads past its arrays: an id
 * outside 1..rows / 1..cols, a malformed line or fewer than nnz entries
 * return GBK_INVALID_VALUE (the error text names the first bad line); blank
 * lines and '%' lines between entries are skipped.  A .gbkcsr path loads the
 * cache as gbk_matrix_load_csr.  vtype: GBK_F32 or GBK_I32. */
int gbk_matrix_create_from_file(gbk_matrix* out, const char* path, gbk_dtype vtype, void* stream);

/* CSR cache: a 64-byte header ("GBKCSR01", int64 rows, cols, nnz, int32
 * value type) then int32 row pointers (rows + 1), int32 column ids (nnz) and
 * 4-byte values (nnz), all little-endian.  Saving reads the CSR back from
 * the device; loading uploads it (the optimised format is not stored). */
int gbk_matrix_save_csr(gbk_matrix A, const char* path, void* stream);
int gbk_matrix_load_csr(gbk_matrix* out, const char* path, void* stream);

/* Copy A's CSR into caller host buffers: row_ptr (rows + 1 int32), col (nnz
 * int32), val (nnz 4-byte values of A's type); any pointer may be NULL. */
int gbk_matrix_download_csr(gbk_matrix A, int32_t* row_ptr, int32_t* col, void* val, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GBK_INGEST_H */
