/* Shared enums of the gbk C ABI.  Numeric values mirror the reference's own
 * enums where one exists, so a shim can pass them through unchanged. */
#ifndef GBK_TYPES_H
#define GBK_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: 0..13 equal LA_Info (src/cpp_graphblas/types.hpp:56-88). */
typedef enum gbk_status {
    GBK_SUCCESS = 0,
    GBK_NO_VALUE = 1,
    GBK_UNINITIALIZED_OBJECT = 2,
    GBK_INVALID_OBJECT = 3,
    GBK_NULL_POINTER = 4,
    GBK_INVALID_VALUE = 5,
    GBK_INVALID_INDEX = 6,
    GBK_DOMAIN_MISMATCH = 7,
    GBK_DIMENSION_MISMATCH = 8,
    GBK_OUTPUT_NOT_EMPTY = 9,
    GBK_OUT_OF_MEMORY = 10,
    GBK_INSUFFICIENT_SPACE = 11,
    GBK_INDEX_OUT_OF_BOUNDS = 12,
    GBK_PANIC = 13,
    /* beyond LA_Info */
    GBK_CUDA_ERROR = 20,  /* a CUDA runtime call failed; text in gbk_get_last_error */
    GBK_UNSUPPORTED = 21, /* operator / type combination not provided */
    GBK_TIMEOUT = 22      /* a bounded device-side wait gave up */
} gbk_status;

/* Element types of vectors and matrix values. */
typedef enum gbk_dtype {
    GBK_F32 = 0,
    GBK_I32 = 1,
    GBK_BOOL = 2, /* one byte, 0 or 1 */
    GBK_I64 = 3,
    GBK_F64 = 4
} gbk_dtype;

/* Storage formats: values equal MatrixStorageFormat
 * (src/helpers/cmd_parser/parser_options.h:16-24). */
typedef enum gbk_format {
    GBK_FMT_CSR = 0,
    GBK_FMT_CSR_SEG = 3,
    GBK_FMT_LAV = 4,
    GBK_FMT_SELL_C = 6
} gbk_format;

/* Semirings of src/cpp_graphblas/types.hpp:274-284 (REGISTER_SEMIRING):
 * add monoid, multiply op, add identity. */
typedef enum gbk_semiring {
    GBK_PLUS_TIMES = 0,      /* PlusMultipliesSemiring     (+, *, 0)            */
    GBK_LOR_LAND = 1,        /* LogicalOrAndSemiring       (||, &&, false)      */
    GBK_FIRST_WINS = 2,      /* FirstWinsSemiring          (first, *, 0)        */
    GBK_FIRST_MIN = 3,       /* FirstMinSemiring           (min, *, 0)          */
    GBK_PLUS_SECOND = 4,     /* PlusSecondSemiring         (+, second, 0)       */
    GBK_STRUCTURAL_BOOL = 5, /* StructuralBool             (||, one, false)     */
    GBK_MIN_PLUS = 6,        /* MinimumPlusSemiring        (min, +, max)        */
    GBK_CUSTOM_LESS_PLUS = 7,/* CustomLessPlusSemiring     (<, +, max)          */
    GBK_MIN_SECOND = 8,      /* MinimumSelectSecondSemiring(min, second, max)   */
    GBK_MIN_NOTEQ = 9,       /* MinimumNotEqualToSemiring  (min, !=, max)       */
    GBK_PLUS_ONE = 10        /* PlusOneSemiring            (+, one, 0)          */
} gbk_semiring;

/* Binary operators (accumulators and element-wise ops), types.hpp:93-192. */
typedef enum gbk_binop {
    GBK_OP_SECOND = 0, /* also "no accumulator" (GrB_NULL -> second, operations.hpp:364-374) */
    GBK_OP_FIRST = 1,
    GBK_OP_PLUS = 2,
    GBK_OP_MINUS = 3,
    GBK_OP_TIMES = 4,
    GBK_OP_DIV = 5,
    GBK_OP_MIN = 6,
    GBK_OP_MAX = 7,
    GBK_OP_LOR = 8,
    GBK_OP_LAND = 9,
    GBK_OP_NE = 10,
    GBK_OP_LT = 11,
    GBK_OP_ONE = 12
} gbk_binop;

/* Unary operators used by apply(). */
typedef enum gbk_unop { GBK_UOP_IDENTITY = 0, GBK_UOP_ABS = 1, GBK_UOP_ONE = 2 } gbk_unop;

/* Monoids of reduce() (REGISTER_MONOID, types.hpp:208-214). */
typedef enum gbk_monoid {
    GBK_MONOID_PLUS = 0,
    GBK_MONOID_MIN = 1,
    GBK_MONOID_MAX = 2,
    GBK_MONOID_LOR = 3,
    GBK_MONOID_LAND = 4
} gbk_monoid;

/* Mask modes: values equal Desc_value (types.hpp:31-38). */
typedef enum gbk_mask_mode {
    GBK_MASK_SCMP = 0,
    GBK_MASK_COMP = 2,
    GBK_MASK_STRUCTURE = 4,
    GBK_MASK_STR_COMP = 5,
    GBK_MASK_DEFAULT = 6
} gbk_mask_mode;

#ifdef __cplusplus
}
#endif
#endif
