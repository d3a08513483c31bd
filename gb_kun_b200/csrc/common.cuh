// Shared device-side vocabulary: semirings, binary operators, cache-hinted
// loads/stores and the error plumbing of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <float.h>
#include <limits.h>
#include <type_traits>

#include "gbk_types.h"

namespace gbk {

// ----------------------------------------------------------------------------
// errors

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define GBK_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t _e = (call);                                                    \
        if (_e != cudaSuccess) return ::gbk::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define GBK_LAUNCH_CHECK()                                                          \
    do {                                                                            \
        cudaError_t _e = cudaGetLastError();                                        \
        if (_e != cudaSuccess) return ::gbk::cuda_fail(_e, "kernel launch", __FILE__, __LINE__); \
    } while (0)

#define GBK_REQUIRE(cond, code, ...)   \
    do {                               \
        if (!(cond)) {                 \
            ::gbk::set_error(__VA_ARGS__); \
            return (code);             \
        }                              \
    } while (0)

int num_sms();
void count_launch(int n);
// Loads the allocation-free conversion's module and caches its scratch
// address for `device` (current); noalloc.cu.
int noalloc_setup(int device);

// Every kernel launch site calls this once the launch is issued.
#define GBK_LAUNCHED()                \
    do {                              \
        ::gbk::count_launch(1);       \
        GBK_LAUNCH_CHECK();           \
    } while (0)

// ----------------------------------------------------------------------------
// cache-hinted global memory access

// Streamed once (matrix arrays): evict-first, no L1 allocation.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
    return __ldcs(p);
}

// L2 eviction policies created per use (createpolicy, PTX ISA 7.4+): the
// gathered vector x is marked evict-last so the matrix stream does not push
// it out of L2.  An instruction-level hint: no device setting is changed.
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float ld_keep(const float* p, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int32_t ld_keep(const int32_t* p, uint64_t pol) {
    int32_t v;
    asm volatile("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
// Re-used across CTAs (x gathers): read-only path, kept in L2.
template <typename T>
__device__ __forceinline__ T ld_reuse(const T* p) {
    return __ldg(p);
}
template <typename T>
__device__ __forceinline__ void st_stream(T* p, T v) {
    __stcs(p, v);
}

// ----------------------------------------------------------------------------
// element types

template <typename T> struct Lim;
template <> struct Lim<float> {
    __host__ __device__ static constexpr float max() { return FLT_MAX; }
};
template <> struct Lim<int32_t> {
    __host__ __device__ static constexpr int32_t max() { return INT_MAX; }
};

// Saturating add for integers: INT_MAX (the min-plus identity) stays infinite.
__device__ __forceinline__ int32_t elem_add(int32_t a, int32_t b) {
    long long s = (long long)a + (long long)b;
    s = s > INT_MAX ? INT_MAX : s;
    s = s < INT_MIN ? INT_MIN : s;
    return (int32_t)s;
}
__device__ __forceinline__ float elem_add(float a, float b) { return a + b; }
__device__ __forceinline__ int64_t elem_add(int64_t a, int64_t b) { return a + b; }
__device__ __forceinline__ double elem_add(double a, double b) { return a + b; }

// ----------------------------------------------------------------------------
// semirings (src/cpp_graphblas/types.hpp:274-284): identity / add / mul,
// mul(A_ij, x_j) with the matrix value first as in spmv_csr.h:366-377.

template <int SR, typename T> struct Semiring;

template <typename T> struct Semiring<GBK_PLUS_TIMES, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return elem_add(a, b); }
    __device__ static T mul(T a, T x) { return a * x; }
};
template <typename T> struct Semiring<GBK_LOR_LAND, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return (a != T(0) || b != T(0)) ? T(1) : T(0); }
    __device__ static T mul(T a, T x) { return (a != T(0) && x != T(0)) ? T(1) : T(0); }
};
template <typename T> struct Semiring<GBK_FIRST_WINS, T> {  // first() is not associative with 0
    static constexpr bool assoc = false;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return a; }
    __device__ static T mul(T a, T x) { return a * x; }
};
template <typename T> struct Semiring<GBK_FIRST_MIN, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return b < a ? b : a; }
    __device__ static T mul(T a, T x) { return a * x; }
};
template <typename T> struct Semiring<GBK_PLUS_SECOND, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return elem_add(a, b); }
    __device__ static T mul(T, T x) { return x; }
};
template <typename T> struct Semiring<GBK_STRUCTURAL_BOOL, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return (a != T(0) || b != T(0)) ? T(1) : T(0); }
    __device__ static T mul(T, T) { return T(1); }
};
template <typename T> struct Semiring<GBK_MIN_PLUS, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return Lim<T>::max(); }
    __device__ static T add(T a, T b) { return b < a ? b : a; }
    __device__ static T mul(T a, T x) { return elem_add(a, x); }
};
template <typename T> struct Semiring<GBK_CUSTOM_LESS_PLUS, T> {  // less() is not associative
    static constexpr bool assoc = false;
    __host__ __device__ static T identity() { return Lim<T>::max(); }
    __device__ static T add(T a, T b) { return a < b ? T(1) : T(0); }
    __device__ static T mul(T a, T x) { return elem_add(a, x); }
};
template <typename T> struct Semiring<GBK_MIN_SECOND, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return Lim<T>::max(); }
    __device__ static T add(T a, T b) { return b < a ? b : a; }
    __device__ static T mul(T, T x) { return x; }
};
template <typename T> struct Semiring<GBK_MIN_NOTEQ, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return Lim<T>::max(); }
    __device__ static T add(T a, T b) { return b < a ? b : a; }
    __device__ static T mul(T a, T x) { return a != x ? T(1) : T(0); }
};
template <typename T> struct Semiring<GBK_PLUS_ONE, T> {
    static constexpr bool assoc = true;
    __host__ __device__ static T identity() { return T(0); }
    __device__ static T add(T a, T b) { return elem_add(a, b); }
    __device__ static T mul(T, T) { return T(1); }
};

// Host-side probe add(3, 5) used by the reference to pick the SpMSpV kernel
// (src/backend/spmspv/spmspv.h:117-146): 8 -> atomic add, 1 -> store 1,
// otherwise a generic read-modify-write.
int semiring_probe(int sr, int dtype);

// Atomic folds of a semiring sum into y (the staged-window kernels).
__device__ __forceinline__ void atomic_min_any(float* p, float v) {
    // order-preserving on the bit patterns: non-negative floats order as ints,
    // negative ones in reverse as unsigned ints
    if (v >= 0.0f)
        atomicMin((int*)p, __float_as_int(v));
    else
        atomicMax((unsigned int*)p, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_min_any(int32_t* p, int32_t v) { atomicMin(p, v); }

// count[key] += 1 for every active lane, one atomic per distinct key in the
// warp (sorted keys repeat within a warp: hub columns, windows)
__device__ __forceinline__ void warp_count(int32_t* count, int32_t key) {
    const unsigned peers = __match_any_sync(__activemask(), key);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(count + key, __popc(peers));
}

__device__ __forceinline__ void atomic_add_any(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_any(int32_t* p, int32_t v) {
    // saturating, like elem_add, so INT_MAX stays the min-plus infinity
    int old = *((volatile int*)p), assumed;
    do {
        assumed = old;
        old = atomicCAS(p, assumed, elem_add(assumed, v));
    } while (old != assumed);
}

// ----------------------------------------------------------------------------
// binary operators (accumulators), runtime-selected: applied once per output.

template <typename T>
__device__ __forceinline__ T binop(int op, T a, T b) {
    switch (op) {
        case GBK_OP_SECOND: return b;
        case GBK_OP_FIRST: return a;
        case GBK_OP_PLUS: return elem_add(a, b);
        case GBK_OP_MINUS: return a - b;
        case GBK_OP_TIMES: return a * b;
        case GBK_OP_DIV:
            if constexpr (std::is_integral<T>::value) return b == T(0) ? T(0) : T(a / b);
            else return a / b;
        case GBK_OP_MIN: return b < a ? b : a;
        case GBK_OP_MAX: return b > a ? b : a;
        case GBK_OP_LOR: return (a != T(0) || b != T(0)) ? T(1) : T(0);
        case GBK_OP_LAND: return (a != T(0) && b != T(0)) ? T(1) : T(0);
        case GBK_OP_NE: return a != b ? T(1) : T(0);
        case GBK_OP_LT: return a < b ? T(1) : T(0);
        case GBK_OP_ONE: return T(1);
    }
    return b;
}

// Mask element test: non-zero means "in the mask" (spmv_csr.h:309).
__device__ __forceinline__ bool mask_at(const void* m, int dtype, int64_t i) {
    switch (dtype) {
        case GBK_F32: return ((const float*)m)[i] != 0.0f;
        case GBK_I32: return ((const int32_t*)m)[i] != 0;
        case GBK_BOOL: return ((const uint8_t*)m)[i] != 0;
        case GBK_I64: return ((const int64_t*)m)[i] != 0;
        case GBK_F64: return ((const double*)m)[i] != 0.0;
    }
    return false;
}

// Row selected by a dense mask under a mask mode (spmv_csr.h:291-313):
// only GrB_STR_COMP complements; every other mode uses the mask as is.
__device__ __forceinline__ bool mask_selects(const void* m, int dtype, int mode, int64_t i) {
    bool v = mask_at(m, dtype, i);
    return mode == GBK_MASK_STR_COMP ? !v : v;
}

template <typename T> constexpr int dtype_of_t();
template <> constexpr int dtype_of_t<float>() { return GBK_F32; }
template <> constexpr int dtype_of_t<int32_t>() { return GBK_I32; }

inline size_t dtype_size(int dt) {
    switch (dt) {
        case GBK_F32: return 4;
        case GBK_I32: return 4;
        case GBK_BOOL: return 1;
        case GBK_I64: return 8;
        case GBK_F64: return 8;
    }
    return 0;
}

}  // namespace gbk
