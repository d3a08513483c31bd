// lablas:: operations with the reference's signatures and semantics
// (src/cpp_graphblas/operations.hpp:53-580 over
// src/backend/operations/operations.h:15-484), each running on the GPU
// through the gbk C ABI.  The reference's per-call behaviour is kept:
// which representation each operand is read in, when the output switches
// between dense and sparse (convert_if_required), how masks select and
// which operations ignore the accumulator.
#pragma once

#include <type_traits>

#include "descriptor.hpp"
#include "matrix.hpp"
#include "vector.hpp"

#define NULL_TYPE long int

namespace lablas {

namespace detail {

template <typename T>
bool null_any(T const& v) {
    return v == nullptr;
}
template <typename L, typename... R>
bool null_any(L const& l, R const&... r) {
    return l == nullptr || null_any(r...);
}

template <typename Op, typename = void> struct has_ucode : std::false_type {};
template <typename Op> struct has_ucode<Op, std::void_t<decltype(Op::gbk_ucode)>> : std::true_type {};

template <typename Op>
constexpr gbk_dtype op_dtype() {
    return dtype_of<typename Op::op_type>::value;
}

// Accumulator code of a functor (second / plus / minus / ...).
template <typename Accum>
constexpr gbk_binop accum_code() {
    return Accum::gbk_code;
}

template <typename M>
gbk_mask mask_arg(const Vector<M>* m, const Descriptor* desc) {
    return m->as_mask(mask_mode(desc));
}

inline LA_Info done(int rc) { return to_info(rc); }

}  // namespace detail

// Runtime form of the reference's compile-time __DISABLE_SPMSPV__ switch
// (operations.h:162-166): while set, mxv / vxm always take the SpMV path.
inline bool& spmspv_disabled() {
    static thread_local bool v = false;
    return v;
}
struct ScopedDisableSpMSpV {
    bool old;
    ScopedDisableSpMSpV() : old(spmspv_disabled()) { spmspv_disabled() = true; }
    ~ScopedDisableSpMSpV() { spmspv_disabled() = old; }
};

// ---------------------------------------------------------------------------
// element-wise (operations.h:216-341)

/* w[i] = mask[i] ^ op(u[i], v[i]) */
template <typename W, typename M, typename U, typename V, typename BinaryOpTAccum, typename BinaryOpT>
LA_Info eWiseAdd(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, BinaryOpT op, const Vector<U>* u,
                 const Vector<V>* v, Descriptor* desc) {
    (void)accum;
    if (detail::null_any(w, u, v)) return GrB_UNINITIALIZED_OBJECT;
    if (w->size() != u->size() || w->size() != v->size()) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->size() != w->size()) return GrB_DIMENSION_MISMATCH;
    const U* up = u->dense_ptr();
    const V* vp = v->dense_ptr();
    W* wp = w->dense_ptr();
    gbk_mask m{};
    if (mask) m = detail::mask_arg(mask, desc);
    return detail::done(gbk_ewise(ewise_add_code<BinaryOpT>(), detail::op_dtype<BinaryOpT>(), wp, Vector<W>::dtype,
                                  up, Vector<U>::dtype, vp, Vector<V>::dtype, w->size(), mask ? &m : nullptr,
                                  stream()));
}
template <typename W, typename M, typename U, typename V, typename BinaryOpT>
LA_Info eWiseAdd(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, BinaryOpT op, const Vector<U>* u,
                 const Vector<V>* v, Descriptor* desc) {
    return eWiseAdd(w, mask, second<U, W, U>(), op, u, v, desc);
}

/* w[i] = mask[i] ^ op(u[i], v[i]) */
template <typename W, typename M, typename U, typename V, typename BinaryOpTAccum, typename BinaryOpT>
LA_Info eWiseMult(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, BinaryOpT op, const Vector<U>* u,
                  const Vector<V>* v, Descriptor* desc) {
    (void)accum;
    if (detail::null_any(w, u, v)) return GrB_UNINITIALIZED_OBJECT;
    if (w->size() != u->size() || w->size() != v->size()) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->size() != w->size()) return GrB_DIMENSION_MISMATCH;
    const U* up = u->dense_ptr();
    const V* vp = v->dense_ptr();
    W* wp = w->dense_ptr();
    gbk_mask m{};
    if (mask) m = detail::mask_arg(mask, desc);
    return detail::done(gbk_ewise(ewise_mul_code<BinaryOpT>(), detail::op_dtype<BinaryOpT>(), wp, Vector<W>::dtype,
                                  up, Vector<U>::dtype, vp, Vector<V>::dtype, w->size(), mask ? &m : nullptr,
                                  stream()));
}
template <typename W, typename M, typename U, typename V, typename BinaryOpT>
LA_Info eWiseMult(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, BinaryOpT op, const Vector<U>* u,
                  const Vector<V>* v, Descriptor* desc) {
    return eWiseMult(w, mask, second<U, W, U>(), op, u, v, desc);
}

namespace detail {
template <typename W, typename M, typename U, typename Op>
LA_Info apply_impl(int kind, Vector<W>* w, const Vector<M>* mask, Op op, double scalar, const Vector<U>* u,
                   Descriptor* desc) {
    (void)op;
    if (null_any(w, u)) return GrB_UNINITIALIZED_OBJECT;
    if (w->size() != u->size()) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->size() != w->size()) return GrB_DIMENSION_MISMATCH;
    const U* up = u->dense_ptr();
    W* wp = w->dense_ptr();
    gbk_mask m{};
    if (mask) m = mask_arg(mask, desc);
    int code;
    if constexpr (has_ucode<Op>::value)
        code = Op::gbk_ucode;
    else
        code = Op::gbk_code;
    return done(gbk_apply(kind, code, op_dtype<Op>(), wp, Vector<W>::dtype, up, Vector<U>::dtype, scalar, w->size(),
                          mask ? &m : nullptr, stream()));
}
}  // namespace detail

/* w[i] = mask[i] ^ op(val, u[i]) */
template <typename W, typename M, typename U, typename T, typename BinaryOpTAccum, typename BinaryOpT>
LA_Info apply(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum, BinaryOpT op, const T val, const Vector<U>* u,
              Descriptor* desc) {
    return detail::apply_impl(1, w, mask, op, (double)val, u, desc);
}
template <typename W, typename M, typename U, typename T, typename BinaryOpT>
LA_Info apply(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, BinaryOpT op, const T val, const Vector<U>* u,
              Descriptor* desc) {
    return detail::apply_impl(1, w, mask, op, (double)val, u, desc);
}
/* w[i] = mask[i] ^ unary_op(u[i]) */
template <typename W, typename M, typename U, typename BinaryOpTAccum, typename UnaryOpT>
LA_Info apply(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum, UnaryOpT op, const Vector<U>* u,
              Descriptor* desc) {
    return detail::apply_impl(0, w, mask, op, 0.0, u, desc);
}
template <typename W, typename M, typename U, typename UnaryOpT>
LA_Info apply(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, UnaryOpT op, const Vector<U>* u, Descriptor* desc) {
    return detail::apply_impl(0, w, mask, op, 0.0, u, desc);
}
/* w[i] = mask[i] ^ op(u[i], val) */
template <typename W, typename M, typename U, typename T, typename BinaryOpTAccum, typename BinaryOpT>
LA_Info apply(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum, BinaryOpT op, const Vector<U>* u, const T val,
              Descriptor* desc) {
    return detail::apply_impl(2, w, mask, op, (double)val, u, desc);
}
template <typename W, typename M, typename U, typename T, typename BinaryOpT>
LA_Info apply(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, BinaryOpT op, const Vector<U>* u, const T val,
              Descriptor* desc) {
    return detail::apply_impl(2, w, mask, op, (double)val, u, desc);
}

// ---------------------------------------------------------------------------
// assign / assignScatter / extract (operations.h:15-147, 401-430)

/* w[indexes[i]] = mask[indexes[i]] ^ value; the accumulator is not used */
template <typename W, typename M, typename U, typename BinaryOpTAccum>
LA_Info assign(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum, U value, const Index* indices, const Index nindices,
               Descriptor* desc) {
    if (w == nullptr) return GrB_UNINITIALIZED_OBJECT;
    if (mask && mask->size() != w->size()) return GrB_DIMENSION_MISMATCH;
    W* wp = w->dense_ptr();
    int rc;
    if (indices) {
        gbk_mask m{};
        if (mask) {
            const_cast<Vector<M>*>(mask)->force_to_dense();  // indexed form reads the dense mask
            m = detail::mask_arg(mask, desc);
        }
        DeviceBuffer<Index> idx(nindices);
        idx.upload(indices, nindices);
        rc = gbk_assign_scalar(wp, Vector<W>::dtype, w->size(), (double)value, mask ? &m : nullptr, idx.p, GBK_I64,
                               nindices, stream());
        cudaStreamSynchronize(current_stream());
    } else {
        gbk_mask m{};
        if (mask) m = detail::mask_arg(mask, desc);
        rc = gbk_assign_scalar(wp, Vector<W>::dtype, w->size(), (double)value, mask ? &m : nullptr, nullptr, GBK_I64,
                               0, stream());
    }
    if (rc) return detail::done(rc);
    w->convert_if_required();
    return GrB_SUCCESS;
}
template <typename W, typename M, typename U>
LA_Info assign(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, U value, const Index* indices, const Index nindices,
               Descriptor* desc) {
    return assign(w, mask, second<U, W, U>(), value, indices, nindices, desc);
}

/* w[i] = accum(w[i], u[i]) under the mask (sparse-mask form: see gbk_assign_vector) */
template <typename W, typename M, typename U, typename BinaryOpTAccum>
LA_Info assign(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, Vector<U>* u, const Index* indices,
               const Index nindices, Descriptor* desc) {
    (void)accum;
    if (w == nullptr) return GrB_UNINITIALIZED_OBJECT;
    if (u == nullptr || w->size() != u->size()) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->size() != w->size()) return GrB_DIMENSION_MISMATCH;
    W* wp = w->dense_ptr();
    const U* up = u->dense_ptr();
    int rc;
    gbk_mask m{};
    if (indices) {
        if (mask) {
            const_cast<Vector<M>*>(mask)->force_to_dense();
            m = detail::mask_arg(mask, desc);
        }
        DeviceBuffer<Index> idx(nindices);
        idx.upload(indices, nindices);
        rc = gbk_assign_vector(detail::accum_code<BinaryOpTAccum>(), Vector<W>::dtype, wp, Vector<W>::dtype, up,
                               Vector<U>::dtype, w->size(), mask ? &m : nullptr, idx.p, GBK_I64, nindices, stream());
        cudaStreamSynchronize(current_stream());
    } else {
        if (mask) m = detail::mask_arg(mask, desc);
        rc = gbk_assign_vector(detail::accum_code<BinaryOpTAccum>(), Vector<W>::dtype, wp, Vector<W>::dtype, up,
                               Vector<U>::dtype, w->size(), mask ? &m : nullptr, nullptr, GBK_I64, 0, stream());
    }
    if (rc) return detail::done(rc);
    w->convert_if_required();
    return GrB_SUCCESS;
}
template <typename W, typename M, typename U>
LA_Info assign(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, Vector<U>* u, const Index* indices,
               const Index nindices, Descriptor* desc) {
    return assign(w, mask, second<U, W, U>(), u, indices, nindices, desc);
}

/* w[indices[k]] = accum(w[indices[k]], u[k]) for k < nindices */
template <typename W, typename M, typename U, typename I, typename BinaryOpTAccum>
LA_Info assignScatter(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, Vector<U>* u,
                      const Vector<I>* indices, const Index nindices, Descriptor* desc) {
    (void)accum;
    if (w == nullptr) return GrB_UNINITIALIZED_OBJECT;
    if (u == nullptr || w->size() != u->size()) return GrB_DIMENSION_MISMATCH;
    W* wp = w->dense_ptr();
    const U* up = u->dense_ptr();
    const I* ip = indices->dense_ptr();
    gbk_mask m{};
    if (mask) {
        const_cast<Vector<M>*>(mask)->force_to_dense();
        m = detail::mask_arg(mask, desc);
    }
    int rc = gbk_assign_vector(detail::accum_code<BinaryOpTAccum>(), Vector<W>::dtype, wp, Vector<W>::dtype, up,
                               Vector<U>::dtype, w->size(), mask ? &m : nullptr, ip, Vector<I>::dtype, nindices,
                               stream());
    if (rc) return detail::done(rc);
    w->convert_if_required();
    return GrB_SUCCESS;
}
template <typename W, typename M, typename U, typename I>
LA_Info assignScatter(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, Vector<U>* u, const Vector<I>* indices,
                      const Index nindices, Descriptor* desc) {
    return assignScatter(w, mask, second<U, W, U>(), u, indices, nindices, desc);
}

/* w[i] = accum(w[i], u[indices[i]]) */
template <typename W, typename M, typename U, typename I, typename BinaryOpT>
LA_Info extract(Vector<W>* w, const Vector<M>* mask, BinaryOpT accum, const Vector<U>* u, const Vector<I>* indices,
                Descriptor* desc) {
    (void)accum;
    if (u == nullptr || w == nullptr || indices == nullptr || desc == nullptr) return GrB_UNINITIALIZED_OBJECT;
    W* wp = w->dense_ptr();
    const U* up = u->dense_ptr();
    gbk_mask m{};
    if (mask) {
        const_cast<Vector<M>*>(mask)->force_to_dense();
        m = detail::mask_arg(mask, desc);
    }
    const I* ip = indices->dense_ptr();
    int rc = gbk_extract(detail::accum_code<BinaryOpT>(), Vector<W>::dtype, wp, Vector<W>::dtype, up,
                         Vector<U>::dtype, w->size(), mask ? &m : nullptr, ip, Vector<I>::dtype, indices->size(),
                         stream());
    if (rc) return detail::done(rc);
    w->convert_if_required();
    return GrB_SUCCESS;
}
template <typename W, typename M, typename U, typename I>
LA_Info extract(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, const Vector<U>* u, const Vector<I>* indices,
                Descriptor* desc) {
    return extract(w, mask, second<U, W, U>(), u, indices, desc);
}

// ---------------------------------------------------------------------------
// mxv / vxm (operations.h:152-211): dense input -> SpMV, sparse -> SpMSpV

namespace detail {

// dst = (D) src on the device, keeping src's current form (dense, or the
// sparse id list with cast values).
template <typename D, typename S>
void cast_into(Vector<D>* dst, const Vector<S>* src) {
    auto* s = const_cast<Vector<S>*>(src);
    if (s->is_dense()) {
        const S* sp = s->dense_ptr();
        throw_if(gbk_vec_cast(sp, Vector<S>::dtype, dst->dense_ptr(), Vector<D>::dtype, s->size(), stream()),
                 "cast");
    } else {
        const Index nv = s->sparse_nvals();
        const int32_t* ids = s->ids_ptr();
        const S* vals = s->vals_ptr();
        dst->adopt_sparse(ids, nv, [&](D* out) {
            throw_if(gbk_vec_cast(vals, Vector<S>::dtype, out, Vector<D>::dtype, nv, stream()), "cast");
        });
    }
}

template <typename W, typename M, typename A, typename U, typename BinaryOpTAccum, typename SemiringT>
LA_Info mxv_same_type(int transpose, Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum, SemiringT,
                      const Matrix<A>* mat, const Vector<U>* u, Descriptor* desc);

// mxv / vxm with element types that differ from the matrix's (the
// reference's templates take W, M, a, U independently,
// src/cpp_graphblas/operations.hpp:347-405): u and w are staged in the
// matrix's element type on the device, the product runs there, and the
// result is cast back into w.  Exact for the integer / boolean semirings;
// a float semiring computes in the matrix's type.
template <typename W, typename M, typename A, typename U, typename BinaryOpTAccum, typename SemiringT>
LA_Info mxv_impl(int transpose, Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, SemiringT op,
                 const Matrix<A>* mat, const Vector<U>* u, Descriptor* desc) {
    if constexpr (std::is_same<W, A>::value && std::is_same<U, A>::value) {
        return mxv_same_type(transpose, w, mask, accum, op, mat, u, desc);
    } else {
        Vector<A> ua(u->size());
        Vector<A> wa(w->size());
        cast_into(&ua, u);
        cast_into(&wa, w);
        LA_Info rc = mxv_same_type(transpose, &wa, mask, accum, op, mat, &ua, desc);
        if (rc != GrB_SUCCESS) return rc;
        cast_into(w, &wa);
        return GrB_SUCCESS;
    }
}

template <typename W, typename M, typename A, typename U, typename BinaryOpTAccum, typename SemiringT>
LA_Info mxv_same_type(int transpose, Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum, SemiringT,
                      const Matrix<A>* mat, const Vector<U>* u, Descriptor* desc) {
    const gbk_semiring sr = SemiringT::gbk_sr;
    const gbk_binop acc = accum_code<BinaryOpTAccum>();
    const Desc_value mode = mask_mode(desc);
    bool dense_input = u->is_dense() || spmspv_disabled();
#ifdef __DISABLE_SPMSPV__
    dense_input = true;
#endif
    int rc;
    if (dense_input) {
        const U* x = u->dense_ptr();
        W* y = w->dense_ptr();
        if (!mask) {
            rc = gbk_mxv(mat->handle(), transpose, sr, acc, Vector<W>::dtype, x, y, nullptr, GBK_BOOL,
                         GBK_MASK_DEFAULT, stream());
        } else if (mask->is_dense()) {
            rc = gbk_mxv(mat->handle(), transpose, sr, acc, Vector<W>::dtype, x, y, mask->dense_ptr(),
                         Vector<M>::dtype, (gbk_mask_mode)mode, stream());
        } else {
            auto* mm = const_cast<Vector<M>*>(mask);
            rc = gbk_mxv_sparse_mask(mat->handle(), transpose, sr, acc, Vector<W>::dtype, x, y, mm->ids_ptr(),
                                     mm->sparse_nvals(), (gbk_mask_mode)mode, stream());
        }
    } else {
        auto* uu = const_cast<Vector<U>*>(u);
        const int32_t* ids = uu->ids_ptr();
        const U* vals = uu->vals_ptr();
        const Index nf = uu->sparse_nvals();
        W* y = w->dense_ptr();
        gbk_mask m{};
        if (mask) m = mask_arg(mask, desc);
        rc = gbk_spmspv(mat->handle(), transpose, sr, acc, Vector<W>::dtype, ids, vals, nf, y, mask ? &m : nullptr,
                        stream());
    }
    if (rc) return done(rc);
    w->convert_if_required();
    return GrB_SUCCESS;
}
}  // namespace detail

template <typename W, typename M, typename a, typename U, typename BinaryOpTAccum, typename SemiringT>
LA_Info mxv(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, SemiringT op, const Matrix<a>* A,
            const Vector<U>* u, Descriptor* desc) {
    if (detail::null_any(w, u, A, desc)) return GrB_UNINITIALIZED_OBJECT;
    return detail::mxv_impl(0, w, mask, accum, op, A, u, desc);
}
template <typename W, typename M, typename a, typename U, typename SemiringT>
LA_Info mxv(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, SemiringT op, const Matrix<a>* A, const Vector<U>* u,
            Descriptor* desc) {
    return mxv(w, mask, second<U, W, U>(), op, A, u, desc);
}

template <typename W, typename M, typename a, typename U, typename BinaryOpTAccum, typename SemiringT>
LA_Info vxm(Vector<W>* w, const Vector<M>* mask, BinaryOpTAccum accum, SemiringT op, const Vector<U>* u,
            const Matrix<a>* A, Descriptor* desc) {
    if (detail::null_any(w, u, A, desc)) return GrB_UNINITIALIZED_OBJECT;
    return detail::mxv_impl(1, w, mask, accum, op, A, u, desc);
}
template <typename W, typename M, typename a, typename U, typename SemiringT>
LA_Info vxm(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, SemiringT op, const Vector<U>* u, const Matrix<a>* A,
            Descriptor* desc) {
    return vxm(w, mask, second<U, W, U>(), op, u, A, desc);
}

// ---------------------------------------------------------------------------
// mxm: masked SpGEMM C<M> = A (+.x) B (operations.h:434-484)

template <typename c, typename m, typename a, typename b, typename BinaryOpT, typename SemiringT>
LA_Info mxm(Matrix<c>* C, const Matrix<m>* mask, BinaryOpT accum, SemiringT op, const Matrix<a>* A,
            const Matrix<b>* B, Descriptor* desc) {
    (void)accum;
    (void)op;
    if (detail::null_any(C, A, B, desc)) return GrB_UNINITIALIZED_OBJECT;
    Desc_value mm = mask_mode(desc);
    if (mm == GrB_COMP || mm == GrB_STR_COMP) throw "Error: complementary mask is not supported yet";
    gbk_matrix out = nullptr;
    if (!mask) {  // unmasked: SpMSpM_unmasked_ikj (spmspm_hash_based_gustavson.h:9-148)
        if (!std::is_same<c, a>::value || !std::is_same<a, b>::value) return GrB_DOMAIN_MISMATCH;
        int rc = gbk_mxm(&out, A->handle(), B->handle(), SemiringT::gbk_sr, stream());
        if (rc) return detail::done(rc);
        return C->adopt_handle(out);
    }
    int rc = gbk_mxm_masked(&out, mask->handle(), A->handle(), B->handle(), SemiringT::gbk_sr,
                            dtype_of<c>::value, stream());
    if (rc) return detail::done(rc);
    std::vector<c> none;
    return C->adopt(out, mask->host_row_ptr(), mask->host_col(), std::move(none));
}
template <typename c, typename m, typename a, typename b, typename SemiringT>
LA_Info mxm(Matrix<c>* C, const Matrix<m>* mask, NULL_TYPE, SemiringT op, const Matrix<a>* A, const Matrix<b>* B,
            Descriptor* desc) {
    return mxm(C, mask, second<c, a, b>(), op, A, B, desc);
}

// ---------------------------------------------------------------------------
// select (select.h): tagged index-unary operators only (lablas::TrilSelect,
// TriuSelect, DiagSelect, OffdiagSelect, Value*Select); a generic callable
// cannot run on the device.

/* Matrix: same structure as u, values op(u_ij, i, j, val) (select.h:363-395,
 * which accumulates into 0, so the accumulator and the mask do not act). */
namespace detail {
// A generic C++ callable (a lambda, as in the reference's
// algorithms/tc/tc.hpp:55-70) is host code and cannot run on the device;
// there is no host fallback, so such a select throws when it is called.
[[noreturn]] inline void select_needs_tagged_operator() {
    throw "Error: select with a generic callable cannot run on the device; use lablas::TrilSelect, TriuSelect, "
          "DiagSelect, OffdiagSelect or ValueEq/Ne/Gt/Ge/Lt/LeSelect";
}
}  // namespace detail

template <typename W, typename M, typename U, typename T, typename BinaryOpT, typename SelectOpT>
LA_Info select(Matrix<W>* w, const Matrix<M>* mask, BinaryOpT accum, SelectOpT op, const Matrix<U>* u, const T val,
               Descriptor* desc) {
    static_assert(std::is_same<W, U>::value, "select keeps the value type of u");
    (void)mask;
    (void)accum;
    (void)op;
    (void)desc;
    if (detail::null_any(w, u)) return GrB_UNINITIALIZED_OBJECT;
    if constexpr (!is_select_op<SelectOpT>::value) {
        detail::select_needs_tagged_operator();
    } else {
        gbk_matrix out = nullptr;
        int rc = gbk_select_matrix(&out, u->handle(), SelectOpT::gbk_sel, (double)val, stream());
        if (rc) return detail::done(rc);
        return w->adopt_handle(out);
    }
}
template <typename W, typename M, typename U, typename T, typename SelectOpT>
LA_Info select(Matrix<W>* w, const Matrix<M>* mask, NULL_TYPE, SelectOpT op, const Matrix<U>* u, const T val,
               Descriptor* desc) {
    return select(w, mask, second<W, U, W>(), op, u, val, desc);
}

namespace detail {
template <typename SelectOpT, typename W, typename M, typename U, typename T, typename BinaryOpT>
LA_Info select_vector_tagged(Vector<W>* w, const Vector<M>* mask, BinaryOpT, const Vector<U>* u, const T val,
                             Descriptor* desc) {
    if (w->size() != u->size()) return GrB_DIMENSION_MISMATCH;
    if (mask && mask->size() != w->size()) return GrB_DIMENSION_MISMATCH;
    const U* up = u->dense_ptr();
    W* wp = w->dense_ptr();
    gbk_mask m{};
    if (mask) m = detail::mask_arg(mask, desc);
    Desc_value out_mode = GrB_DEFAULT;
    if (desc) desc->get(GrB_OUTPUT, &out_mode);
    return detail::done(gbk_select_vector(SelectOpT::gbk_sel, (double)val, wp, Vector<W>::dtype, up,
                                          Vector<U>::dtype, w->size(), BinaryOpT::gbk_code, mask ? &m : nullptr,
                                          mask && out_mode == GrB_REPLACE, stream()));
}
}  // namespace detail

/* Vector: w[i] = accum(w[i], op(u[i], i, 0, val)) where the mask selects;
 * GrB_REPLACE zeroes the rest (select.h:17-315). */
template <typename W, typename M, typename U, typename T, typename BinaryOpT, typename SelectOpT>
LA_Info select(Vector<W>* w, const Vector<M>* mask, BinaryOpT accum, SelectOpT op, const Vector<U>* u, const T val,
               Descriptor* desc) {
    (void)accum;
    (void)op;
    if (detail::null_any(w, u)) return GrB_UNINITIALIZED_OBJECT;
    if constexpr (!is_select_op<SelectOpT>::value) {
        detail::select_needs_tagged_operator();
    } else {
        return detail::select_vector_tagged<SelectOpT>(w, mask, accum, u, val, desc);
    }
}

template <typename W, typename M, typename U, typename T, typename SelectOpT>
LA_Info select(Vector<W>* w, const Vector<M>* mask, NULL_TYPE, SelectOpT op, const Vector<U>* u, const T val,
               Descriptor* desc) {
    return select(w, mask, second<W, U, W>(), op, u, val, desc);
}

// ---------------------------------------------------------------------------
// reduce (operations.h:346-396)

template <typename T, typename U, typename BinaryOpTAccum, typename MonoidT>
LA_Info reduce(T* val, BinaryOpTAccum accum, MonoidT op, const Vector<U>* u, Descriptor* desc) {
    (void)desc;
    if (u == nullptr) return GrB_UNINITIALIZED_OBJECT;
    static_assert(MonoidT::gbk_monoid_code >= 0, "reduce runs plus / min / max / or monoids on the device");
    typedef typename MonoidT::op_type R;
    R r = op.identity();
    int rc;
    auto* uu = const_cast<Vector<U>*>(u);
    if (uu->is_dense())
        rc = gbk_reduce((gbk_monoid)MonoidT::gbk_monoid_code, dtype_of<R>::value, uu->dense_ptr(), Vector<U>::dtype,
                        uu->size(), &r, stream());
    else
        rc = gbk_reduce((gbk_monoid)MonoidT::gbk_monoid_code, dtype_of<R>::value, uu->vals_ptr(), Vector<U>::dtype,
                        uu->sparse_nvals(), &r, stream());
    if (rc) return detail::done(rc);
    *val = accum(*val, r);
    return GrB_SUCCESS;
}
template <typename T, typename U, typename MonoidT>
LA_Info reduce(T* val, NULL_TYPE, MonoidT op, const Vector<U>* u, Descriptor* desc) {
    return reduce(val, second<T, T, T>(), op, u, desc);
}

template <typename T, typename U, typename BinaryOpTAccum, typename MonoidT>
LA_Info reduce(T* val, BinaryOpTAccum accum, MonoidT op, const Matrix<U>* u, Descriptor* desc) {
    (void)desc;
    if (u == nullptr) return GrB_UNINITIALIZED_OBJECT;
    typedef typename MonoidT::op_type R;
    R r = op.identity();
    const int32_t* p;
    const int32_t* i;
    const void* v;
    int rc = gbk_matrix_csr_arrays(u->handle(), 0, &p, &i, &v, stream());
    if (rc) return detail::done(rc);
    rc = gbk_reduce((gbk_monoid)MonoidT::gbk_monoid_code, dtype_of<R>::value, v, Matrix<U>::dtype, u->get_nnz(), &r,
                    stream());
    if (rc) return detail::done(rc);
    *val = accum(*val, r);
    return GrB_SUCCESS;
}
template <typename T, typename U, typename MonoidT>
LA_Info reduce(T* val, NULL_TYPE, MonoidT op, const Matrix<U>* u, Descriptor* desc) {
    return reduce(val, second<T, T, T>(), op, u, desc);
}

}  // namespace lablas
