// lablas:: operator vocabulary: the reference's functors, monoids and
// semirings (src/cpp_graphblas/types.hpp:93-349) with the same names and
// host semantics, each tagged with the gbk C-ABI code that runs it on the GPU.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <limits>
#include <type_traits>

#include "gbk.h"

typedef long long Index;
#define VNT Index
#define ENT Index

enum Storage { GrB_UNKNOWN, GrB_SPARSE, GrB_DENSE };

enum Desc_field {
    GrB_MASK,
    GrB_OUTPUT,
    GrB_INP0,
    GrB_INP1,
    GrB_MODE,
    GrB_TA,
    GrB_TB,
    GrB_NT,
    GrB_MXVMODE,
    GrB_TOL,
    GrB_BACKEND,
    GrB_MXMMODE,
    GrB_NDESCFIELD
};

enum Desc_value {
    GrB_SCMP = 0,
    GrB_REPLACE = 1,
    GrB_COMP = 2,
    GrB_TRAN = 3,
    GrB_STRUCTURE = 4,
    GrB_STR_COMP = 5,
    GrB_DEFAULT = 6,
    GrB_FIXEDROW,
    GrB_PUSHPULL = 10,
    GrB_PUSHONLY = 11,
    GrB_PULLONLY = 12,
    GrB_SEQUENTIAL = 13,
    GrB_CUDA = 14,
    GrB_8 = 8,
    GrB_16 = 16,
    GrB_32 = 32,
    GrB_64 = 64,
    GrB_128 = 128,
    GrB_256 = 256,
    GrB_512 = 512,
    GrB_1024 = 1024,
    GrB_IJK = 20,
    GrB_IKJ = 21,
    GrB_IKJ_MASKED = 22,
    GrB_IJK_DOUBLE_SORT = 23
};

typedef enum {
    GrB_SUCCESS = 0,
    GrB_NO_VALUE = 1,
    GrB_UNINITIALIZED_OBJECT = 2,
    GrB_INVALID_OBJECT = 3,
    GrB_NULL_POINTER = 4,
    GrB_INVALID_VALUE = 5,
    GrB_INVALID_INDEX = 6,
    GrB_DOMAIN_MISMATCH = 7,
    GrB_DIMENSION_MISMATCH = 8,
    GrB_OUTPUT_NOT_EMPTY = 9,
    GrB_OUT_OF_MEMORY = 10,
    GrB_INSUFFICIENT_SPACE = 11,
    GrB_INDEX_OUT_OF_BOUNDS = 12,
    GrB_PANIC = 13
} LA_Info;

enum MatrixStorageFormat { CSR = 0, COO = 1, CSR_SEG = 3, LAV = 4, VECT_GROUP_CSR = 5, SELL_C = 6, SORTED_CSR = 7 };

namespace lablas {

// element type -> gbk_dtype
template <typename T> struct dtype_of;
template <> struct dtype_of<float> { static constexpr gbk_dtype value = GBK_F32; };
template <> struct dtype_of<double> { static constexpr gbk_dtype value = GBK_F64; };
template <> struct dtype_of<int> { static constexpr gbk_dtype value = GBK_I32; };
template <> struct dtype_of<bool> { static constexpr gbk_dtype value = GBK_BOOL; };
template <> struct dtype_of<long long> { static constexpr gbk_dtype value = GBK_I64; };
template <> struct dtype_of<long> { static constexpr gbk_dtype value = GBK_I64; };

// ---------------------------------------------------------------------------
// binary / unary operators (types.hpp:93-192)

#define GBK_BINOP(NAME, CODE, EXPR)                                                       \
    template <typename T_in1, typename T_in2 = T_in1, typename T_out = T_in1>            \
    struct NAME {                                                                         \
        static constexpr gbk_binop gbk_code = CODE;                                       \
        typedef T_in1 op_type;                                                            \
        typedef T_out out_type;                                                           \
        inline T_out operator()(const T_in1 lhs, const T_in2 rhs) const { return EXPR; } \
    };

GBK_BINOP(plus, GBK_OP_PLUS, lhs + rhs)
GBK_BINOP(minus, GBK_OP_MINUS, lhs - rhs)
GBK_BINOP(multiplies, GBK_OP_TIMES, lhs * rhs)
GBK_BINOP(first, GBK_OP_FIRST, lhs)
GBK_BINOP(second, GBK_OP_SECOND, rhs)
GBK_BINOP(minimum, GBK_OP_MIN, (rhs < lhs) ? rhs : lhs)
GBK_BINOP(maximum, GBK_OP_MAX, (rhs > lhs) ? rhs : lhs)
GBK_BINOP(GrB_ONEB_T, GBK_OP_ONE, (T_out)1)
#undef GBK_BINOP

template <typename T_in1, typename T_in2 = T_in1, typename T_out = T_in1>
struct not_equal_to {
    static constexpr gbk_binop gbk_code = GBK_OP_NE;
    typedef T_in1 op_type;
    typedef T_out out_type;
    inline T_out operator()(T_in1 lhs, T_in2 rhs) const { return lhs != rhs; }
};
template <typename T_in1 = bool, typename T_in2 = bool, typename T_out = bool>
struct logical_and {
    static constexpr gbk_binop gbk_code = GBK_OP_LAND;
    typedef T_in1 op_type;
    typedef T_out out_type;
    inline T_out operator()(const T_in1 lhs, const T_in2 rhs) const { return lhs && rhs; }
};
template <typename T_in1 = bool, typename T_in2 = bool, typename T_out = bool>
struct logical_or {
    static constexpr gbk_binop gbk_code = GBK_OP_LOR;
    typedef T_in1 op_type;
    typedef T_out out_type;
    inline T_out operator()(const T_in1 lhs, const T_in2 rhs) const { return lhs || rhs; }
};
template <typename T_in1, typename T_in2 = T_in1, typename T_out = bool>
struct less {
    static constexpr gbk_binop gbk_code = GBK_OP_LT;
    typedef T_in1 op_type;
    typedef T_out out_type;
    inline T_out operator()(T_in1 lhs, T_in2 rhs) const { return lhs < rhs; }
};
template <typename T>
struct div {
    static constexpr gbk_binop gbk_code = GBK_OP_DIV;
    typedef T op_type;
    typedef T out_type;
    inline T operator()(const T lhs, const T rhs) const { return lhs / rhs; }
};
template <typename T_out>
struct abs {
    static constexpr gbk_unop gbk_ucode = GBK_UOP_ABS;
    typedef T_out op_type;
    inline T_out operator()(const T_out arg) const { return std::abs(arg); }
};
template <typename D1, typename D2 = D1>
struct Identity {
    static constexpr gbk_unop gbk_ucode = GBK_UOP_IDENTITY;
    typedef D1 op_type;
    inline D2 operator()(const D1 input) const { return input; }
};

// ---------------------------------------------------------------------------
// monoids (REGISTER_MONOID, types.hpp:208-214)

#define GBK_MONOID(NAME, BINOP, IDENT, MCODE)                                            \
    template <typename T_out>                                                             \
    struct NAME {                                                                         \
        static constexpr gbk_binop gbk_code = BINOP<T_out>::gbk_code;                     \
        static constexpr int gbk_monoid_code = MCODE;                                     \
        typedef T_out op_type;                                                            \
        inline T_out identity() const { return static_cast<T_out>(IDENT); }               \
        inline T_out operator()(T_out lhs, T_out rhs) const { return BINOP<T_out>()(lhs, rhs); } \
    };

GBK_MONOID(PlusMonoid, plus, 0, GBK_MONOID_PLUS)
GBK_MONOID(LogicalOrMonoid, logical_or, false, GBK_MONOID_LOR)
GBK_MONOID(MinimumMonoid, minimum, std::numeric_limits<T_out>::max(), GBK_MONOID_MIN)
GBK_MONOID(FirstWinsMonoid, first, 0, -1)
GBK_MONOID(SecondWinsMonoid, second, 0, -1)
GBK_MONOID(CustomLessMonoid, less, std::numeric_limits<T_out>::max(), -1)
GBK_MONOID(FirstMin, minimum, 0, GBK_MONOID_MIN)
#undef GBK_MONOID

// ---------------------------------------------------------------------------
// semirings (REGISTER_SEMIRING, types.hpp:274-284)

template <typename Add, typename Mul, gbk_semiring Code>
struct SemiringBase {
    static constexpr gbk_semiring gbk_sr = Code;
    static constexpr gbk_binop gbk_add = Add::gbk_code;
    static constexpr gbk_binop gbk_mul = Mul::gbk_code;
};

#define GBK_SEMIRING(NAME, ADD_MONOID, MUL_OP, CODE)                                          \
    template <typename T_in1, typename T_in2 = T_in1, typename T_out = T_in1>                \
    struct NAME : SemiringBase<ADD_MONOID<T_out>, MUL_OP<T_in1, T_in2, T_out>, CODE> {        \
        typedef T_out result_type;                                                            \
        typedef T_out T_out_type;                                                             \
        typedef T_in1 op_type;                                                                \
        inline T_out identity() const { return ADD_MONOID<T_out>().identity(); }              \
        inline T_out add_op(T_out lhs, T_out rhs) const { return ADD_MONOID<T_out>()(lhs, rhs); } \
        inline T_out mul_op(T_in1 lhs, T_in2 rhs) const { return MUL_OP<T_in1, T_in2, T_out>()(lhs, rhs); } \
    };

GBK_SEMIRING(PlusMultipliesSemiring, PlusMonoid, multiplies, GBK_PLUS_TIMES)
GBK_SEMIRING(LogicalOrAndSemiring, LogicalOrMonoid, logical_and, GBK_LOR_LAND)
GBK_SEMIRING(FirstWinsSemiring, FirstWinsMonoid, multiplies, GBK_FIRST_WINS)
GBK_SEMIRING(FirstMinSemiring, FirstMin, multiplies, GBK_FIRST_MIN)
GBK_SEMIRING(PlusSecondSemiring, PlusMonoid, second, GBK_PLUS_SECOND)
GBK_SEMIRING(StructuralBool, LogicalOrMonoid, GrB_ONEB_T, GBK_STRUCTURAL_BOOL)
GBK_SEMIRING(MinimumPlusSemiring, MinimumMonoid, plus, GBK_MIN_PLUS)
GBK_SEMIRING(CustomLessPlusSemiring, CustomLessMonoid, plus, GBK_CUSTOM_LESS_PLUS)
GBK_SEMIRING(MinimumSelectSecondSemiring, MinimumMonoid, second, GBK_MIN_SECOND)
GBK_SEMIRING(MinimumNotEqualToSemiring, MinimumMonoid, not_equal_to, GBK_MIN_NOTEQ)
GBK_SEMIRING(PlusOneSemiring, PlusMonoid, GrB_ONEB_T, GBK_PLUS_ONE)
#undef GBK_SEMIRING

// eWiseAdd takes a semiring's add monoid, eWiseMult its multiply operator,
// and a plain operator as is (generic_extract_add / _mull, types.hpp:255-272).
template <typename T, typename = void> struct is_semiring : std::false_type {};
template <typename T> struct is_semiring<T, std::void_t<decltype(T::gbk_sr)>> : std::true_type {};

// Index-unary select operators (the GraphBLAS GrB_TRIL ... GrB_VALUELE
// family), tagged with their C-ABI code: op(x, i, j, k) returns x where the
// operator keeps the entry and 0 where not, the convention of the
// reference's select lambdas (algorithms/tc/tc.hpp:55-70).
#define GBK_SELECT_OP(NAME, CODE, KEEP)                                                         \
    template <typename T>                                                                      \
    struct NAME {                                                                              \
        static constexpr gbk_select_op gbk_sel = CODE;                                         \
        inline T operator()(T x, long long i, long long j, double k) const {                   \
            (void)i;                                                                           \
            (void)j;                                                                           \
            return (KEEP) ? x : T(0);                                                          \
        }                                                                                      \
    };
GBK_SELECT_OP(TrilSelect, GBK_SEL_TRIL, (double)j <= (double)i + k)
GBK_SELECT_OP(TriuSelect, GBK_SEL_TRIU, (double)j >= (double)i + k)
GBK_SELECT_OP(DiagSelect, GBK_SEL_DIAG, (double)j == (double)i + k)
GBK_SELECT_OP(OffdiagSelect, GBK_SEL_OFFDIAG, (double)j != (double)i + k)
GBK_SELECT_OP(ValueEqSelect, GBK_SEL_VALUE_EQ, (double)x == k)
GBK_SELECT_OP(ValueNeSelect, GBK_SEL_VALUE_NE, (double)x != k)
GBK_SELECT_OP(ValueGtSelect, GBK_SEL_VALUE_GT, (double)x > k)
GBK_SELECT_OP(ValueGeSelect, GBK_SEL_VALUE_GE, (double)x >= k)
GBK_SELECT_OP(ValueLtSelect, GBK_SEL_VALUE_LT, (double)x < k)
GBK_SELECT_OP(ValueLeSelect, GBK_SEL_VALUE_LE, (double)x <= k)
#undef GBK_SELECT_OP

template <typename T, typename = void> struct is_select_op : std::false_type {};
template <typename T> struct is_select_op<T, std::void_t<decltype(T::gbk_sel)>> : std::true_type {};

template <typename Op> constexpr gbk_binop ewise_add_code() {
    if constexpr (is_semiring<Op>::value) return Op::gbk_add;
    else return Op::gbk_code;
}
template <typename Op> constexpr gbk_binop ewise_mul_code() {
    if constexpr (is_semiring<Op>::value) return Op::gbk_mul;
    else return Op::gbk_code;
}

}  // namespace lablas
