// GrB_* C-style wrappers, LAGraph_Graph and the operator / descriptor macros
// the algorithm ports use (src/cblas_wrappers/{types,operations,
// vector_methods,matrix_methods}.hpp), over the device lablas:: API.
#pragma once

#include <cstdio>
#include <string>

#include "operations.hpp"

#define GrB_Index Index
#define GrB_ALL NULL
#define GrB_NULL ((long int)NULL)

template <typename T>
struct LAGraph_Graph {
    lablas::Matrix<T>* A;
    lablas::Matrix<T>* AT;  // the reference aliases AT to A (cblas_wrappers/types.hpp:21-22)
    lablas::Vector<GrB_Index>* rowdegree;
    lablas::Vector<GrB_Index>* coldegree;

    explicit LAGraph_Graph(lablas::Matrix<T>& m) {
        Index nrows, ncols;
        m.get_nrows(&nrows);
        m.get_ncols(&ncols);
        A = &m;
        AT = &m;
        rowdegree = new lablas::Vector<Index>(nrows);
        coldegree = new lablas::Vector<Index>(ncols);
        rowdegree->build(m.get_rowdegrees(), nrows);
        coldegree->build(m.get_coldegrees(), ncols);
    }
    ~LAGraph_Graph() {
        delete rowdegree;
        delete coldegree;
    }
};

#define GrB_TRY(CallInstruction)                                                                         \
    {                                                                                                   \
        LA_Info code = CallInstruction;                                                                 \
        if (code != GrB_SUCCESS) printf("GraphBLAS error: %d at call \"" #CallInstruction "\"\n", (int)code); \
    }

#define LG_CLEAR_MSG

enum GrB_Type { GrB_FP32 = 0, GrB_BOOL = 1, GrB_INT32 = 2, GrB_INT64 = 3 };

// binary operations
#define GrB_DIV_FP32 lablas::div<float>()
#define GrB_MAX_FP32 lablas::maximum<float, float, float>()
#define GrB_PLUS_FP32 lablas::plus<float>()
#define GrB_MINUS_FP32 lablas::minus<float>()
#define GrB_ABS_FP32 lablas::abs<float>()
#define GrB_SECOND_INT64 lablas::second<long long int>()
#define GrB_SECOND_INT32 lablas::second<int>()
#define GrB_SECOND_FLT32 lablas::second<float>()

// semirings
#define LAGraph_plus_second_fp32 lablas::PlusSecondSemiring<float>()
#define LAGraph_structural_bool lablas::StructuralBool<bool>()
#define LAGraph_plus_one_int64 lablas::PlusOneSemiring<long long>()

// monoids
#define GrB_PLUS_MONOID_FP32 lablas::PlusMonoid<float>()
#define GrB_PLUS_MONOID_INT32 lablas::PlusMonoid<int>()
#define GrB_PLUS_MONOID_INT64 lablas::PlusMonoid<long long>()

// descriptors
#define GrB_DESC_RSC (&lablas::GrB_DESC_RSC)
#define GrB_DESC_C (&lablas::GrB_DESC_C)
#define GrB_DESC_S (&lablas::GrB_DESC_S)
#define GrB_DESC_SC (&lablas::GrB_DESC_SC)

// ---- vectors / matrices (vector_methods.hpp, matrix_methods.hpp) ----

template <typename T>
LA_Info GrB_Vector_new(lablas::Vector<T>** v, GrB_Type, GrB_Index size, const std::string& name = "unknown") {
    *v = new lablas::Vector<T>(size);
    (*v)->set_name(name);
    return GrB_SUCCESS;
}
template <typename T>
LA_Info GrB_free(lablas::Vector<T>** v) {
    delete *v;
    *v = nullptr;
    return GrB_SUCCESS;
}
template <typename W, typename T>
LA_Info GrB_Vector_setElement(lablas::Vector<W>* w, const T val, GrB_Index index) {
    return w->set_element(val, index);
}
template <typename W>
LA_Info GrB_Vector_nvals(Index* nvals, const lablas::Vector<W>* w) {
    return w->get_nvals(nvals);
}
template <typename T>
LA_Info GrB_Vector_clear(lablas::Vector<T>* v) {
    return v->clear();
}
template <typename T>
LA_Info GrB_Matrix_new(lablas::Matrix<T>** m, GrB_Type, GrB_Index, GrB_Index) {
    *m = new lablas::Matrix<T>();
    return GrB_SUCCESS;
}
template <typename T>
LA_Info GrB_free(lablas::Matrix<T>** m) {
    delete *m;
    *m = nullptr;
    return GrB_SUCCESS;
}
template <typename T>
LA_Info GrB_Matrix_nrows(GrB_Index* n, lablas::Matrix<T>* m) {
    return m->get_nrows(n);
}
template <typename T>
LA_Info GrB_Matrix_cols(GrB_Index* n, lablas::Matrix<T>* m) {
    return m->get_ncols(n);
}
template <typename T>
LA_Info GrB_Matrix_nvals(GrB_Index* n, lablas::Matrix<T>* m) {
    return m->get_nvals(n);
}

// ---- operations (cblas_wrappers/operations.hpp:5-228) ----

template <typename W, typename M, typename U, typename T, typename A, typename Op>
LA_Info GrB_apply(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, Op op, const T val,
                  const lablas::Vector<U>* u, lablas::Descriptor* desc) {
    return lablas::apply(w, mask, accum, op, val, u, desc);
}
template <typename W, typename M, typename U, typename A, typename Op>
LA_Info GrB_apply(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, Op op, const lablas::Vector<U>* u,
                  lablas::Descriptor* desc) {
    return lablas::apply(w, mask, accum, op, u, desc);
}
template <typename W, typename M, typename U, typename T, typename A, typename Op>
LA_Info GrB_apply(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, Op op, const lablas::Vector<U>* u,
                  const T val, lablas::Descriptor* desc) {
    return lablas::apply(w, mask, accum, op, u, val, desc);
}
template <typename W, typename M, typename U, typename A>
LA_Info GrB_assign(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, U value, const GrB_Index* indices,
                   const GrB_Index nindices, lablas::Descriptor* desc) {
    return lablas::assign(w, mask, accum, value, indices, nindices, desc);
}
template <typename W, typename M, typename U, typename A>
LA_Info GrB_assign(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, lablas::Vector<U>* u,
                   const GrB_Index* indices, const GrB_Index nindices, lablas::Descriptor* desc) {
    return lablas::assign(w, mask, accum, u, indices, nindices, desc);
}
template <typename W, typename M, typename U, typename V, typename A, typename Op>
LA_Info GrB_eWiseAdd(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, Op op, const lablas::Vector<U>* u,
                     const lablas::Vector<V>* v, lablas::Descriptor* desc) {
    return lablas::eWiseAdd(w, mask, accum, op, u, v, desc);
}
template <typename W, typename M, typename U, typename V, typename A, typename Op>
LA_Info GrB_eWiseMult(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, Op op,
                      const lablas::Vector<U>* u, const lablas::Vector<V>* v, lablas::Descriptor* desc) {
    return lablas::eWiseMult(w, mask, accum, op, u, v, desc);
}
template <typename W, typename M, typename a, typename U, typename A, typename S>
LA_Info GrB_vxm(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, S op, const lablas::Vector<U>* u,
                const lablas::Matrix<a>* m, lablas::Descriptor* desc) {
    return lablas::vxm(w, mask, accum, op, u, m, desc);
}
template <typename W, typename M, typename a, typename U, typename A, typename S>
LA_Info GrB_mxv(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, S op, const lablas::Matrix<a>* m,
                const lablas::Vector<U>* u, lablas::Descriptor* desc) {
    return lablas::mxv(w, mask, accum, op, m, u, desc);
}
template <typename W, typename M, typename a, typename U, typename A, typename S>
LA_Info GrB_mxm(lablas::Matrix<W>* c, const lablas::Matrix<M>* mask, A accum, S op, const lablas::Matrix<U>* a_,
                const lablas::Matrix<a>* b, lablas::Descriptor* desc) {
    return lablas::mxm(c, mask, accum, op, a_, b, desc);
}
// GrB_select (src/cblas_wrappers/operations.hpp:189-230): tagged operators only (lablas::TrilSelect, ...)
template <typename W, typename M, typename U, typename T, typename A, typename S>
LA_Info GrB_select(lablas::Vector<W>* w, const lablas::Vector<M>* mask, A accum, S op, const lablas::Vector<U>* u,
                   const T val, lablas::Descriptor* desc) {
    return lablas::select(w, mask, accum, op, u, val, desc);
}
template <typename W, typename M, typename U, typename T, typename A, typename S>
LA_Info GrB_select(lablas::Matrix<W>* w, const lablas::Matrix<M>* mask, A accum, S op, const lablas::Matrix<U>* u,
                   const T val, lablas::Descriptor* desc) {
    return lablas::select(w, mask, accum, op, u, val, desc);
}
template <typename T, typename U, typename A, typename Mon>
LA_Info GrB_reduce(T* val, A accum, Mon op, const lablas::Vector<U>* u, lablas::Descriptor* desc) {
    return lablas::reduce(val, accum, op, u, desc);
}
template <typename T, typename U, typename A, typename Mon>
LA_Info GrB_reduce(T* val, A accum, Mon op, const lablas::Matrix<U>* u, lablas::Descriptor* desc) {
    return lablas::reduce(val, accum, op, u, desc);
}
