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
} gbk_format_params;

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

#ifdef __cplusplus
}
#endif
#endif
