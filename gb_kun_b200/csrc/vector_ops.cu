// Element-wise vector operations, dense <-> sparse conversion and reductions.
//
// These are the per-iteration O(n) steps of the algorithms (assign, eWise,
// apply, extract, reduce: src/backend/operations/operations.h:15-430 with
// generic_operations.h / indexed_operations.h).  They are HBM-streaming
// kernels: one thread per element, grid-stride, values converted on load to
// the operator's type and on store to the output type.  Mask semantics
// follow the reference exactly, including its choice of which index reads u
// for sparse masks (noted per entry point in include/gbk.h).
#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace gbk {

namespace {

template <typename OT>
__device__ __forceinline__ OT ld_as(const void* p, int dt, int64_t i) {
    switch (dt) {
        case GBK_F32: return (OT)((const float*)p)[i];
        case GBK_I32: return (OT)((const int32_t*)p)[i];
        case GBK_BOOL: return (OT)(((const uint8_t*)p)[i] != 0);
        case GBK_I64: return (OT)((const int64_t*)p)[i];
        case GBK_F64: return (OT)((const double*)p)[i];
    }
    return OT(0);
}

template <typename OT>
__device__ __forceinline__ void st_as(void* p, int dt, int64_t i, OT v) {
    switch (dt) {
        case GBK_F32: ((float*)p)[i] = (float)v; return;
        case GBK_I32: ((int32_t*)p)[i] = (int32_t)v; return;
        case GBK_BOOL: ((uint8_t*)p)[i] = (v != OT(0)) ? 1 : 0; return;
        case GBK_I64: ((int64_t*)p)[i] = (int64_t)v; return;
        case GBK_F64: ((double*)p)[i] = (double)v; return;
    }
}

template <typename T>
__device__ __forceinline__ T binop_any(int op, T a, T b) {
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

template <typename T>
__device__ __forceinline__ T unop_any(int op, T a) {
    switch (op) {
        case GBK_UOP_IDENTITY: return a;
        case GBK_UOP_ABS: return a < T(0) ? T(-a) : a;
        case GBK_UOP_ONE: return T(1);
    }
    return a;
}

// Which positions a dense mask selects for assign (generic_operations.h:52-59).
__device__ __forceinline__ bool assign_selects(bool m, int mode) {
    return (!m && mode == GBK_MASK_STR_COMP) || (m && (mode == GBK_MASK_DEFAULT || mode == GBK_MASK_STRUCTURE));
}

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    int64_t cap = (int64_t)num_sms() * 16;
    if (b > cap) b = cap;
    return (unsigned)(b > 0 ? b : 1);
}

#define GRID_LOOP(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------
// kernels

__global__ void k_flag_nonzero(const void* v, int dt, int64_t n, int32_t* flag) {
    GRID_LOOP(i, n) flag[i] = ld_as<double>(v, dt, i) != 0.0 ? 1 : 0;
}

__global__ void k_compact(const void* v, int dt, int64_t n, const int32_t* pos, const int32_t* flag, int32_t* ids,
                          void* vals) {
    GRID_LOOP(i, n) {
        if (flag[i]) {
            int32_t p = pos[i];
            ids[p] = (int32_t)i;
            switch (dt) {
                case GBK_F32: ((float*)vals)[p] = ((const float*)v)[i]; break;
                case GBK_I32: ((int32_t*)vals)[p] = ((const int32_t*)v)[i]; break;
                case GBK_BOOL: ((uint8_t*)vals)[p] = ((const uint8_t*)v)[i]; break;
                case GBK_I64: ((int64_t*)vals)[p] = ((const int64_t*)v)[i]; break;
                case GBK_F64: ((double*)vals)[p] = ((const double*)v)[i]; break;
            }
        }
    }
}

__global__ void k_scatter_vals(const int32_t* ids, const void* vals, int64_t nvals, int dt, void* dense) {
    GRID_LOOP(k, nvals) {
        int32_t i = ids[k];
        switch (dt) {
            case GBK_F32: ((float*)dense)[i] = ((const float*)vals)[k]; break;
            case GBK_I32: ((int32_t*)dense)[i] = ((const int32_t*)vals)[k]; break;
            case GBK_BOOL: ((uint8_t*)dense)[i] = ((const uint8_t*)vals)[k]; break;
            case GBK_I64: ((int64_t*)dense)[i] = ((const int64_t*)vals)[k]; break;
            case GBK_F64: ((double*)dense)[i] = ((const double*)vals)[k]; break;
        }
    }
}

template <typename OT>
__global__ void k_fill(void* v, int dt, int64_t n, OT value) {
    GRID_LOOP(i, n) st_as<OT>(v, dt, i, value);
}

__global__ void k_iota(void* v, int dt, int64_t n) {
    GRID_LOOP(i, n) st_as<int64_t>(v, dt, i, i);
}

__global__ void k_cast(const void* src, int st, void* dst, int dt, int64_t n) {
    GRID_LOOP(i, n) {
        if (dt == GBK_F64 || st == GBK_F64 || dt == GBK_F32 || st == GBK_F32)
            st_as<double>(dst, dt, i, ld_as<double>(src, st, i));
        else
            st_as<int64_t>(dst, dt, i, ld_as<int64_t>(src, st, i));
    }
}

// mask form selector for element-wise kernels: 0 none, 1 dense, 2 sparse
template <typename OT>
__global__ void k_ewise(int op, void* w, int wt, const void* u, int ut, const void* v, int vt, int64_t n,
                        int mform, const void* mdense, int mdt, const int32_t* mids, int64_t mnv) {
    const int64_t cnt = (mform == 2) ? mnv : n;
    GRID_LOOP(k, cnt) {
        int64_t i = k;
        if (mform == 2) i = mids[k];
        else if (mform == 1 && !mask_at(mdense, mdt, i)) continue;
        st_as<OT>(w, wt, i, binop_any<OT>(op, ld_as<OT>(u, ut, i), ld_as<OT>(v, vt, i)));
    }
}

template <typename OT>
__global__ void k_apply(int kind, int op, void* w, int wt, const void* u, int ut, OT scalar, int64_t n, int mform,
                        const void* mdense, int mdt, const int32_t* mids, int64_t mnv) {
    const int64_t cnt = (mform == 2) ? mnv : n;
    GRID_LOOP(k, cnt) {
        int64_t i = k;
        if (mform == 2) i = mids[k];
        else if (mform == 1 && !mask_at(mdense, mdt, i)) continue;
        OT a = ld_as<OT>(u, ut, i);
        OT r = kind == 0 ? unop_any<OT>(op, a) : (kind == 1 ? binop_any<OT>(op, scalar, a) : binop_any<OT>(op, a, scalar));
        st_as<OT>(w, wt, i, r);
    }
}

// Scalar assign over all positions / a dense mask (mode-aware) / ids.
template <typename OT>
__global__ void k_assign_scalar(void* w, int wt, int64_t n, OT value, int mform, const void* mdense, int mdt,
                                int mmode, const int32_t* mids, int64_t mnv) {
    const int64_t cnt = (mform == 2) ? mnv : n;
    GRID_LOOP(k, cnt) {
        int64_t i = k;
        if (mform == 2) i = mids[k];
        else if (mform == 1 && !assign_selects(mask_at(mdense, mdt, i), mmode)) continue;
        st_as<OT>(w, wt, i, value);
    }
}

template <typename OT>
__global__ void k_assign_scalar_idx(void* w, int wt, OT value, const void* idx, int it, int64_t nidx,
                                    const void* mdense, int mdt) {
    GRID_LOOP(k, nidx) {
        int64_t i = ld_as<int64_t>(idx, it, k);
        if (mdense && !mask_at(mdense, mdt, i)) continue;
        st_as<OT>(w, wt, i, value);
    }
}

// w[i] = accum(w[i], u[j]) forms of vector assign / extract
// mode 0: i = j = k (k over n), dense mask tested with `sel` rule
// mode 1: i = ids[k], j = k (sparse mask quirk of assign)
// mode 2: i = k, j = ids[k] (sparse mask quirk of extract)
template <typename OT>
__global__ void k_accum_map(int accum, void* w, int wt, const void* u, int ut, int64_t n, int mode, int sel_rule,
                            const void* mdense, int mdt, int mmode, const int32_t* mids, int64_t mnv) {
    const int64_t cnt = (mode == 0) ? n : mnv;
    GRID_LOOP(k, cnt) {
        int64_t i = k, j = k;
        if (mode == 1) i = mids[k];
        if (mode == 2) j = mids[k];
        if (mode == 0 && mdense) {
            bool m = mask_at(mdense, mdt, k);
            bool s = sel_rule ? assign_selects(m, mmode) : m;
            if (!s) continue;
        }
        st_as<OT>(w, wt, i, binop_any<OT>(accum, ld_as<OT>(w, wt, i), ld_as<OT>(u, ut, j)));
    }
}

// Sparse STR_COMP masks: expand to a dense 0/1 byte mask.
__global__ void k_mark_ids(const int32_t* ids, int64_t nv, uint8_t* flag) {
    GRID_LOOP(k, nv) flag[ids[k]] = 1;
}

// assignScatter with sequential-order resolution of repeated indices.
__global__ void k_scatter_winner(const void* idx, int it, int64_t nidx, const void* mdense, int mdt, int32_t* win) {
    GRID_LOOP(k, nidx) {
        int64_t i = ld_as<int64_t>(idx, it, k);
        if (mdense && !mask_at(mdense, mdt, i)) continue;
        atomicMax(&win[i], (int32_t)k);
    }
}

template <typename OT>
__global__ void k_scatter_apply(int accum, void* w, int wt, const void* u, int ut, const void* idx, int it,
                                int64_t nidx, const int32_t* win) {
    GRID_LOOP(k, nidx) {
        int64_t i = ld_as<int64_t>(idx, it, k);
        if (win[i] != (int32_t)k) continue;
        st_as<OT>(w, wt, i, binop_any<OT>(accum, ld_as<OT>(w, wt, i), ld_as<OT>(u, ut, k)));
    }
}

template <typename OT>
__global__ void k_gather(int accum, void* w, int wt, const void* u, int ut, const void* idx, int it, int64_t nidx,
                         const void* mdense, int mdt) {
    GRID_LOOP(i, nidx) {
        int64_t j = ld_as<int64_t>(idx, it, i);
        if (mdense && !mask_at(mdense, mdt, j)) continue;
        st_as<OT>(w, wt, i, binop_any<OT>(accum, ld_as<OT>(w, wt, i), ld_as<OT>(u, ut, j)));
    }
}

template <typename AT>
__device__ __forceinline__ AT monoid_apply(int m, AT a, AT b) {
    switch (m) {
        case GBK_MONOID_PLUS: return a + b;
        case GBK_MONOID_MIN: return b < a ? b : a;
        case GBK_MONOID_MAX: return b > a ? b : a;
        case GBK_MONOID_LOR: return (a != AT(0) || b != AT(0)) ? AT(1) : AT(0);
        case GBK_MONOID_LAND: return (a != AT(0) && b != AT(0)) ? AT(1) : AT(0);
    }
    return a;
}

// Two-pass deterministic reduction: fixed grid of partials, then one block.
template <typename AT>
__global__ void k_reduce_partial(int m, AT ident, const void* u, int ut, int64_t n, AT* part) {
    __shared__ AT sh[kThreads];
    AT acc = ident;
    GRID_LOOP(i, n) acc = monoid_apply<AT>(m, acc, ld_as<AT>(u, ut, i));
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = monoid_apply<AT>(m, sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

template <typename AT>
__global__ void k_reduce_final(int m, AT ident, const AT* part, int np, AT* out) {
    __shared__ AT sh[kThreads];
    AT acc = ident;
    for (int i = threadIdx.x; i < np; i += kThreads) acc = monoid_apply<AT>(m, acc, part[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = monoid_apply<AT>(m, sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

bool is_float(int dt) { return dt == GBK_F32 || dt == GBK_F64; }

struct MaskArgs {
    int form = 0;  // 0 none, 1 dense, 2 sparse
    const void* dense = nullptr;
    int dtype = 0;
    int mode = GBK_MASK_DEFAULT;
    const int32_t* ids = nullptr;
    int64_t nvals = 0;
};

MaskArgs mask_args(const gbk_mask* m) {
    MaskArgs a;
    if (!m) return a;
    a.mode = m->mode;
    if (m->dense) {
        a.form = 1;
        a.dense = m->dense;
        a.dtype = m->dtype;
    } else {
        a.form = 2;
        a.ids = m->ids;
        a.nvals = m->nvals;
    }
    return a;
}

// Dispatch on the operator type.
#define OPTYPE_SWITCH(ot, BODY)                         \
    switch (ot) {                                       \
        case GBK_F32: { using OT = float; BODY; } break; \
        case GBK_I32: { using OT = int32_t; BODY; } break; \
        case GBK_BOOL: { using OT = int32_t; BODY; } break; \
        case GBK_I64: { using OT = int64_t; BODY; } break; \
        case GBK_F64: { using OT = double; BODY; } break; \
        default: set_error("bad operator type %d", (int)(ot)); return GBK_INVALID_VALUE; \
    }

}  // namespace

// Dense byte mask from a sparse id list (scratch allocated on the stream).
static int expand_sparse_mask(const MaskArgs& m, int64_t n, uint8_t** out, cudaStream_t s) {
    uint8_t* flag = nullptr;
    GBK_CUDA(cudaMallocAsync((void**)&flag, n > 0 ? n : 1, s));
    GBK_CUDA(cudaMemsetAsync(flag, 0, n > 0 ? n : 1, s));
    if (m.nvals > 0) {
        k_mark_ids<<<grid_for(m.nvals), kThreads, 0, s>>>(m.ids, m.nvals, flag);
        GBK_LAUNCHED();
    }
    *out = flag;
    return GBK_SUCCESS;
}

}  // namespace gbk

using namespace gbk;

extern "C" {

int gbk_vec_nvals(const void* v, gbk_dtype t, int64_t n, int64_t* out, void* stream) {
    GBK_REQUIRE(v || n == 0, GBK_NULL_POINTER, "gbk_vec_nvals: NULL vector");
    GBK_REQUIRE(out, GBK_NULL_POINTER, "gbk_vec_nvals: NULL out");
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        *out = 0;
        return GBK_SUCCESS;
    }
    int32_t* flag = nullptr;
    GBK_CUDA(cudaMallocAsync((void**)&flag, sizeof(int32_t) * n, s));
    k_flag_nonzero<<<grid_for(n), kThreads, 0, s>>>(v, t, n, flag);
    GBK_LAUNCHED();
    int64_t r = 0;
    int rc = gbk_reduce(GBK_MONOID_PLUS, GBK_I64, flag, GBK_I32, n, &r, stream);
    cudaFreeAsync(flag, s);
    *out = r;
    return rc;
}

int gbk_vec_to_sparse(const void* dense, gbk_dtype t, int64_t n, int32_t* ids, void* vals, int64_t* nvals,
                      void* stream) {
    GBK_REQUIRE(nvals, GBK_NULL_POINTER, "gbk_vec_to_sparse: NULL nvals");
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        *nvals = 0;
        return GBK_SUCCESS;
    }
    GBK_REQUIRE(dense && ids && vals, GBK_NULL_POINTER, "gbk_vec_to_sparse: NULL array");
    GBK_REQUIRE(n > 0 && n < INT32_MAX, GBK_INVALID_VALUE, "gbk_vec_to_sparse: n = %lld outside [0, 2^31 - 1)",
                (long long)n);
    int32_t *flag = nullptr, *pos = nullptr;
    GBK_CUDA(cudaMallocAsync((void**)&flag, sizeof(int32_t) * (n + 1), s));
    GBK_CUDA(cudaMallocAsync((void**)&pos, sizeof(int32_t) * (n + 1), s));
    GBK_CUDA(cudaMemsetAsync(flag + n, 0, sizeof(int32_t), s));
    k_flag_nonzero<<<grid_for(n), kThreads, 0, s>>>(dense, t, n, flag);
    GBK_LAUNCHED();
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, pos, (int)(n + 1), s);
    void* tmp = nullptr;
    GBK_CUDA(cudaMallocAsync(&tmp, tb, s));
    GBK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, flag, pos, (int)(n + 1), s));
    count_launch(1);
    k_compact<<<grid_for(n), kThreads, 0, s>>>(dense, t, n, pos, flag, ids, vals);
    GBK_LAUNCHED();
    int32_t cnt = 0;
    GBK_CUDA(cudaMemcpyAsync(&cnt, pos + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    cudaFreeAsync(tmp, s);
    cudaFreeAsync(flag, s);
    cudaFreeAsync(pos, s);
    GBK_CUDA(cudaStreamSynchronize(s));
    *nvals = cnt;
    return GBK_SUCCESS;
}

int gbk_vec_to_dense(const int32_t* ids, const void* vals, int64_t nvals, gbk_dtype t, void* dense, int64_t n,
                     void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(dense, GBK_NULL_POINTER, "gbk_vec_to_dense: NULL dense");
    GBK_CUDA(cudaMemsetAsync(dense, 0, dtype_size(t) * n, s));
    if (nvals > 0) {
        GBK_REQUIRE(ids && vals, GBK_NULL_POINTER, "gbk_vec_to_dense: NULL sparse arrays");
        k_scatter_vals<<<grid_for(nvals), kThreads, 0, s>>>(ids, vals, nvals, t, dense);
        GBK_LAUNCHED();
    }
    return GBK_SUCCESS;
}

int gbk_vec_fill(void* v, gbk_dtype t, int64_t n, double value, void* stream) {
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(v, GBK_NULL_POINTER, "gbk_vec_fill: NULL vector");
    cudaStream_t s = (cudaStream_t)stream;
    if (is_float(t))
        k_fill<double><<<grid_for(n), kThreads, 0, s>>>(v, t, n, value);
    else
        k_fill<int64_t><<<grid_for(n), kThreads, 0, s>>>(v, t, n, (int64_t)value);
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

int gbk_vec_iota(void* v, gbk_dtype t, int64_t n, void* stream) {
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(v, GBK_NULL_POINTER, "gbk_vec_iota: NULL vector");
    k_iota<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(v, t, n);
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

int gbk_vec_cast(const void* src, gbk_dtype st, void* dst, gbk_dtype dt, int64_t n, void* stream) {
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(src && dst, GBK_NULL_POINTER, "gbk_vec_cast: NULL vector");
    k_cast<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(src, st, dst, dt, n);
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

int gbk_ewise(gbk_binop op, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut, const void* v,
              gbk_dtype vt, int64_t n, const gbk_mask* mask, void* stream) {
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(w && u && v, GBK_NULL_POINTER, "gbk_ewise: NULL vector");
    MaskArgs m = mask_args(mask);
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t cnt = m.form == 2 ? m.nvals : n;
    if (cnt == 0) return GBK_SUCCESS;
    OPTYPE_SWITCH(optype, (k_ewise<OT><<<grid_for(cnt), kThreads, 0, s>>>(op, w, wt, u, ut, v, vt, n, m.form,
                                                                            m.dense, m.dtype, m.ids, m.nvals)));
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

int gbk_apply(int kind, int op, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut,
              double scalar, int64_t n, const gbk_mask* mask, void* stream) {
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(w && u, GBK_NULL_POINTER, "gbk_apply: NULL vector");
    GBK_REQUIRE(kind >= 0 && kind <= 2, GBK_INVALID_VALUE, "gbk_apply: bad kind %d", kind);
    MaskArgs m = mask_args(mask);
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t cnt = m.form == 2 ? m.nvals : n;
    if (cnt == 0) return GBK_SUCCESS;
    OPTYPE_SWITCH(optype, (k_apply<OT><<<grid_for(cnt), kThreads, 0, s>>>(kind, op, w, wt, u, ut, (OT)scalar, n,
                                                                            m.form, m.dense, m.dtype, m.ids,
                                                                            m.nvals)));
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

int gbk_assign_scalar(void* w, gbk_dtype wt, int64_t n, double value, const gbk_mask* mask, const void* indices,
                      gbk_dtype index_t, int64_t nindices, void* stream) {
    GBK_REQUIRE(w || n == 0, GBK_NULL_POINTER, "gbk_assign_scalar: NULL vector");
    cudaStream_t s = (cudaStream_t)stream;
    MaskArgs m = mask_args(mask);
    if (indices) {
        GBK_REQUIRE(m.form != 2, GBK_INVALID_VALUE, "gbk_assign_scalar: indexed assign needs a dense mask");
        if (nindices == 0) return GBK_SUCCESS;
        if (is_float(wt))
            k_assign_scalar_idx<double><<<grid_for(nindices), kThreads, 0, s>>>(w, wt, value, indices, index_t,
                                                                                nindices, m.dense, m.dtype);
        else
            k_assign_scalar_idx<int64_t><<<grid_for(nindices), kThreads, 0, s>>>(
                w, wt, (int64_t)value, indices, index_t, nindices, m.dense, m.dtype);
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }
    if (n == 0) return GBK_SUCCESS;
    uint8_t* expanded = nullptr;
    if (m.form == 2) {
        if (m.mode == GBK_MASK_STR_COMP) {  // the reference densifies the mask and complements it
            int rc = expand_sparse_mask(m, n, &expanded, s);
            if (rc) return rc;
            m.form = 1;
            m.dense = expanded;
            m.dtype = GBK_BOOL;
        } else if (m.mode != GBK_MASK_DEFAULT && m.mode != GBK_MASK_STRUCTURE) {
            return GBK_SUCCESS;  // COMP / SCMP select nothing (generic_operations.h:26-46)
        }
    }
    const int64_t cnt = m.form == 2 ? m.nvals : n;
    if (cnt > 0) {
        if (is_float(wt))
            k_assign_scalar<double><<<grid_for(cnt), kThreads, 0, s>>>(w, wt, n, value, m.form, m.dense, m.dtype,
                                                                        m.mode, m.ids, m.nvals);
        else
            k_assign_scalar<int64_t><<<grid_for(cnt), kThreads, 0, s>>>(w, wt, n, (int64_t)value, m.form, m.dense,
                                                                         m.dtype, m.mode, m.ids, m.nvals);
        GBK_LAUNCHED();
    }
    if (expanded) cudaFreeAsync(expanded, s);
    return GBK_SUCCESS;
}

int gbk_assign_vector(gbk_binop accum, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut,
                      int64_t n, const gbk_mask* mask, const void* indices, gbk_dtype index_t, int64_t nindices,
                      void* stream) {
    GBK_REQUIRE((w && u) || n == 0, GBK_NULL_POINTER, "gbk_assign_vector: NULL vector");
    cudaStream_t s = (cudaStream_t)stream;
    MaskArgs m = mask_args(mask);
    if (indices) {
        GBK_REQUIRE(m.form != 2, GBK_INVALID_VALUE, "gbk_assign_vector: indexed assign needs a dense mask");
        if (nindices == 0 || n == 0) return GBK_SUCCESS;
        int32_t* win = nullptr;
        GBK_CUDA(cudaMallocAsync((void**)&win, sizeof(int32_t) * n, s));
        GBK_CUDA(cudaMemsetAsync(win, 0xff, sizeof(int32_t) * n, s));  // -1
        k_scatter_winner<<<grid_for(nindices), kThreads, 0, s>>>(indices, index_t, nindices, m.dense, m.dtype, win);
        GBK_LAUNCHED();
        OPTYPE_SWITCH(optype, (k_scatter_apply<OT><<<grid_for(nindices), kThreads, 0, s>>>(
                                  accum, w, wt, u, ut, indices, index_t, nindices, win)));
        GBK_LAUNCHED();
        cudaFreeAsync(win, s);
        return GBK_SUCCESS;
    }
    if (n == 0) return GBK_SUCCESS;
    uint8_t* expanded = nullptr;
    int mode = 0;
    if (m.form == 2) {
        if (m.mode == GBK_MASK_STR_COMP) {
            int rc = expand_sparse_mask(m, n, &expanded, s);
            if (rc) return rc;
            m.form = 1;
            m.dense = expanded;
            m.dtype = GBK_BOOL;
        } else if (m.mode == GBK_MASK_DEFAULT || m.mode == GBK_MASK_STRUCTURE) {
            mode = 1;
        } else {
            return GBK_SUCCESS;
        }
    }
    const int64_t cnt = mode == 1 ? m.nvals : n;
    if (cnt > 0) {
        OPTYPE_SWITCH(optype, (k_accum_map<OT><<<grid_for(cnt), kThreads, 0, s>>>(
                                  accum, w, wt, u, ut, n, mode, 1, m.form == 1 ? m.dense : nullptr, m.dtype, m.mode,
                                  m.ids, m.nvals)));
        GBK_LAUNCHED();
    }
    if (expanded) cudaFreeAsync(expanded, s);
    return GBK_SUCCESS;
}

int gbk_extract(gbk_binop accum, gbk_dtype optype, void* w, gbk_dtype wt, const void* u, gbk_dtype ut, int64_t n,
                const gbk_mask* mask, const void* indices, gbk_dtype index_t, int64_t nindices, void* stream) {
    GBK_REQUIRE((w && u) || n == 0, GBK_NULL_POINTER, "gbk_extract: NULL vector");
    cudaStream_t s = (cudaStream_t)stream;
    MaskArgs m = mask_args(mask);
    if (indices) {
        GBK_REQUIRE(m.form != 2, GBK_INVALID_VALUE, "gbk_extract: indexed extract needs a dense mask");
        if (nindices == 0) return GBK_SUCCESS;
        OPTYPE_SWITCH(optype, (k_gather<OT><<<grid_for(nindices), kThreads, 0, s>>>(
                                  accum, w, wt, u, ut, indices, index_t, nindices, m.dense, m.dtype)));
        GBK_LAUNCHED();
        return GBK_SUCCESS;
    }
    const int mode = m.form == 2 ? 2 : 0;
    const int64_t cnt = mode == 2 ? m.nvals : n;
    if (cnt == 0) return GBK_SUCCESS;
    OPTYPE_SWITCH(optype, (k_accum_map<OT><<<grid_for(cnt), kThreads, 0, s>>>(
                              accum, w, wt, u, ut, n, mode, 0, m.form == 1 ? m.dense : nullptr, m.dtype, m.mode,
                              m.ids, m.nvals)));
    GBK_LAUNCHED();
    return GBK_SUCCESS;
}

int gbk_reduce(gbk_monoid monoid, gbk_dtype rt, const void* u, gbk_dtype ut, int64_t n, void* result,
               void* stream) {
    GBK_REQUIRE(result, GBK_NULL_POINTER, "gbk_reduce: NULL result");
    GBK_REQUIRE((int)monoid >= 0 && (int)monoid <= GBK_MONOID_LAND, GBK_INVALID_VALUE, "gbk_reduce: bad monoid");
    cudaStream_t s = (cudaStream_t)stream;
    const bool fl = is_float(rt) || is_float(ut);
    // identities (types.hpp:208-214)
    double idf = 0.0;
    int64_t idi = 0;
    if (monoid == GBK_MONOID_MIN) {
        idf = rt == GBK_F32 ? (double)FLT_MAX : 1.7976931348623157e308;
        idi = rt == GBK_I32 ? INT_MAX : (rt == GBK_BOOL ? 1 : INT64_MAX);
    } else if (monoid == GBK_MONOID_MAX) {
        idf = rt == GBK_F32 ? -(double)FLT_MAX : -1.7976931348623157e308;
        idi = rt == GBK_I32 ? INT_MIN : (rt == GBK_BOOL ? 0 : INT64_MIN);
    } else if (monoid == GBK_MONOID_LAND) {
        idf = 1.0;
        idi = 1;
    }
    const int np = (int)grid_for(n > 0 ? n : 1);
    void* part = nullptr;
    void* dres = nullptr;
    GBK_CUDA(cudaMallocAsync(&part, 8 * (size_t)np, s));
    GBK_CUDA(cudaMallocAsync(&dres, 8, s));
    if (fl) {
        k_reduce_partial<double><<<np, kThreads, 0, s>>>(monoid, idf, u, ut, n, (double*)part);
        GBK_LAUNCHED();
        k_reduce_final<double><<<1, kThreads, 0, s>>>(monoid, idf, (const double*)part, np, (double*)dres);
        GBK_LAUNCHED();
    } else {
        k_reduce_partial<int64_t><<<np, kThreads, 0, s>>>(monoid, idi, u, ut, n, (int64_t*)part);
        GBK_LAUNCHED();
        k_reduce_final<int64_t><<<1, kThreads, 0, s>>>(monoid, idi, (const int64_t*)part, np, (int64_t*)dres);
        GBK_LAUNCHED();
    }
    union {
        double d;
        int64_t i;
    } hv;
    GBK_CUDA(cudaMemcpyAsync(&hv, dres, 8, cudaMemcpyDeviceToHost, s));
    cudaFreeAsync(part, s);
    cudaFreeAsync(dres, s);
    GBK_CUDA(cudaStreamSynchronize(s));
    switch (rt) {
        case GBK_F32: *(float*)result = fl ? (float)hv.d : (float)hv.i; break;
        case GBK_F64: *(double*)result = fl ? hv.d : (double)hv.i; break;
        case GBK_I32: *(int32_t*)result = fl ? (int32_t)hv.d : (int32_t)hv.i; break;
        case GBK_I64: *(int64_t*)result = fl ? (int64_t)hv.d : hv.i; break;
        case GBK_BOOL: *(uint8_t*)result = fl ? (hv.d != 0.0) : (hv.i != 0); break;
        default: set_error("gbk_reduce: bad result type"); return GBK_INVALID_VALUE;
    }
    return GBK_SUCCESS;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// select (src/backend/operations/select.h)

namespace gbk {
namespace {

// Does the index-unary operator keep an entry with value x at (i, j)?
__device__ __forceinline__ bool select_keeps(int op, int64_t i, int64_t j, double x, double k) {
    const int64_t ki = (int64_t)k;
    switch (op) {
        case GBK_SEL_TRIL: return j <= i + ki;
        case GBK_SEL_TRIU: return j >= i + ki;
        case GBK_SEL_DIAG: return j == i + ki;
        case GBK_SEL_OFFDIAG: return j != i + ki;
        case GBK_SEL_VALUE_EQ: return x == k;
        case GBK_SEL_VALUE_NE: return x != k;
        case GBK_SEL_VALUE_GT: return x > k;
        case GBK_SEL_VALUE_GE: return x >= k;
        case GBK_SEL_VALUE_LT: return x < k;
        case GBK_SEL_VALUE_LE: return x <= k;
    }
    return false;
}

template <typename T>
__global__ void k_select_matrix(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                const T* __restrict__ val, int64_t nrows, int64_t nnz, int op, double k,
                                T* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int64_t lo = 0, hi = nrows;  // row of entry e
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (ptr[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    out[e] = select_keeps(op, lo, idx[e], (double)val[e], k) ? val[e] : T(0);
}

template <typename OT>
__global__ void k_select_vector(int op, double k, void* w, int wt, const void* u, int ut, int64_t n, int accum,
                                const void* mask, int mdt, int comp, int replace) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        bool sel = true;
        if (mask) sel = (ld_as<double>(mask, mdt, i) != 0.0) != (comp != 0);
        if (sel) {
            const OT x = ld_as<OT>(u, ut, i);
            const OT r = select_keeps(op, i, 0, (double)x, k) ? x : OT(0);
            st_as<OT>(w, wt, i, binop_any<OT>(accum, ld_as<OT>(w, wt, i), r));
        } else if (replace) {
            st_as<OT>(w, wt, i, OT(0));
        }
    }
}

}  // namespace
}  // namespace gbk

extern "C" int gbk_select_matrix(gbk_matrix* out, gbk_matrix A, gbk_select_op op, double thunk, void* stream) {
    using namespace gbk;
    GBK_REQUIRE(out && A, GBK_NULL_POINTER, "gbk_select_matrix: NULL argument");
    GBK_REQUIRE(op >= GBK_SEL_TRIL && op <= GBK_SEL_VALUE_LE, GBK_INVALID_VALUE, "gbk_select_matrix: bad operator %d",
                (int)op);
    cudaStream_t s = (cudaStream_t)stream;
    const CsrView& v = A->csr;
    void* vals = nullptr;
    GBK_CUDA(cudaMalloc(&vals, 4 * (v.nnz > 0 ? v.nnz : 1)));
    if (v.nnz > 0) {
        if (A->vtype == GBK_F32)
            k_select_matrix<float><<<(unsigned)((v.nnz + 255) / 256), 256, 0, s>>>(
                v.ptr, v.idx, (const float*)v.val, v.nrows, v.nnz, (int)op, thunk, (float*)vals);
        else
            k_select_matrix<int32_t><<<(unsigned)((v.nnz + 255) / 256), 256, 0, s>>>(
                v.ptr, v.idx, (const int32_t*)v.val, v.nrows, v.nnz, (int)op, thunk, (int32_t*)vals);
        count_launch(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            cudaFree(vals);
            return cuda_fail(e, "select kernel", __FILE__, __LINE__);
        }
    }
    const int rc = gbk_matrix_create_csr(out, v.nrows, v.ncols, v.nnz, v.ptr, v.idx, vals, A->vtype, 1, stream);
    cudaStreamSynchronize(s);
    cudaFree(vals);
    return rc;
}

extern "C" int gbk_select_vector(gbk_select_op op, double thunk, void* w, gbk_dtype wt, const void* u, gbk_dtype ut,
                                 int64_t n, gbk_binop accum, const gbk_mask* mask, int replace, void* stream) {
    using namespace gbk;
    if (n == 0) return GBK_SUCCESS;
    GBK_REQUIRE(w && u, GBK_NULL_POINTER, "gbk_select_vector: NULL vector");
    GBK_REQUIRE(op >= GBK_SEL_TRIL && op <= GBK_SEL_VALUE_LE, GBK_INVALID_VALUE, "gbk_select_vector: bad operator %d",
                (int)op);
    cudaStream_t s = (cudaStream_t)stream;
    MaskArgs m = mask_args(mask);
    uint8_t* expanded = nullptr;
    if (m.form == 2) {  // a sparse mask selects its ids (as a structure)
        int rc = expand_sparse_mask(m, n, &expanded, s);
        if (rc) return rc;
        m.dense = expanded;
        m.dtype = GBK_BOOL;
        m.form = 1;
    }
    const int comp = m.form && (m.mode == GBK_MASK_COMP || m.mode == GBK_MASK_SCMP || m.mode == GBK_MASK_STR_COMP);
    const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 16);
    const int ot = (is_float(wt) || is_float(ut)) ? GBK_F64 : GBK_I64;
    if (ot == GBK_F64)
        k_select_vector<double><<<grid, 256, 0, s>>>((int)op, thunk, w, wt, u, ut, n, (int)accum,
                                                     m.form ? m.dense : nullptr, m.dtype, comp, replace);
    else
        k_select_vector<int64_t><<<grid, 256, 0, s>>>((int)op, thunk, w, wt, u, ut, n, (int)accum,
                                                      m.form ? m.dense : nullptr, m.dtype, comp, replace);
    count_launch(1);
    cudaError_t e = cudaGetLastError();
    if (expanded) cudaFreeAsync(expanded, s);
    if (e != cudaSuccess) return cuda_fail(e, "select kernel", __FILE__, __LINE__);
    return GBK_SUCCESS;
}
