// Triangle counting, Burkhardt's method (algorithms/tc/tc.hpp:88-284, the
// default of LAGr_TriangleCount): C<A> = A (+.one) A counts, for every edge
// (i, j), the common neighbours of i and j; sum(C) / 6 is the number of
// triangles of the symmetric graph A.  gbk_triangle_count gives that number
// without forming C: on a symmetric loop-free A it orients every edge from
// its (degree, id)-smaller end and counts each triangle once (hub rows then
// meet only short lists); any other A takes the masked product as written.
#pragma once

#include <cstdint>

#include "lablas/gb_kun.h"

namespace lablas {
namespace algorithm {

inline uint64_t triangle_count_burkhardt(const Matrix<int>* A) {
    uint64_t ntri = 0;
    throw_if(gbk_triangle_count(A->handle(), &ntri, stream()), "triangle count");
    return ntri;
}

// The same formula through the GraphBLAS calls the reference makes (masked
// plus-one mxm, then reduce).
inline uint64_t triangle_count_burkhardt_mxm(const Matrix<int>* A) {
    Matrix<int> C;
    Descriptor mxm_desc({{GrB_MXMMODE, GrB_IKJ_MASKED}});
    LA_Info rc = mxm(&C, A, GrB_NULL, LAGraph_plus_one_int64, A, A, &mxm_desc);
    if (rc != GrB_SUCCESS) throw "Error: masked mxm failed in triangle counting";
    int64_t ntri = 0;
    rc = reduce(&ntri, GrB_NULL, GrB_PLUS_MONOID_INT64, &C, (Descriptor*)nullptr);
    if (rc != GrB_SUCCESS) throw "Error: reduce failed in triangle counting";
    return (uint64_t)(ntri / 6);
}

// The other methods of LAGr_TriangleCount (algorithms/tc/tc.hpp:219-273)
// with the reference's own prep (tricount_prep, :46-75): its "L" and "U" come
// from select lambdas that zero the values of one triangle but keep every
// entry (select.h:363-395 keeps u's structure), so L = A's structure with the
// values of j >= i (TriuSelect, k = 0) and U = A's structure with the values
// of j <= i (TrilSelect, k = 0).  Each method is then a masked plus-one
// product, which counts structure, divided by 6 as the reference does.
enum TriangleCountMethod {
    TriangleCount_Default = 0,
    TriangleCount_Burkhardt = 1,
    TriangleCount_Cohen = 2,
    TriangleCount_Sandia = 3,
    TriangleCount_Sandia2 = 4,
    TriangleCount_SandiaDot = 5,
    TriangleCount_SandiaDot2 = 6
};

inline uint64_t triangle_count(const Matrix<int>* A, int method) {
    if (method == TriangleCount_Default || method == TriangleCount_Burkhardt) return triangle_count_burkhardt(A);
    if (method < TriangleCount_Cohen || method > TriangleCount_SandiaDot2) throw "Error: unknown triangle count method";
    Matrix<int> L, U, C;
    LA_Info rc = select(&L, (const Matrix<int>*)nullptr, GrB_NULL, TriuSelect<int>(), A, 0, (Descriptor*)nullptr);
    if (rc == GrB_SUCCESS)
        rc = select(&U, (const Matrix<int>*)nullptr, GrB_NULL, TrilSelect<int>(), A, 0, (Descriptor*)nullptr);
    if (rc != GrB_SUCCESS) throw "Error: select failed in triangle counting";
    Descriptor mxm_desc({{GrB_MXMMODE, GrB_IKJ_MASKED}});
    const Matrix<int>* M = A;
    const Matrix<int>* X = &L;
    const Matrix<int>* Y = &U;
    switch (method) {
        case TriangleCount_Cohen: M = A; X = &L; Y = &U; break;       // (L * U) .* A
        case TriangleCount_Sandia: M = &L; X = &L; Y = &L; break;     // (L * L) .* L
        case TriangleCount_Sandia2: M = &U; X = &U; Y = &U; break;    // (U * U) .* U
        case TriangleCount_SandiaDot: M = &L; X = &L; Y = &U; break;  // (L * U) .* L
        case TriangleCount_SandiaDot2: M = &U; X = &U; Y = &L; break; // (U * L) .* U
    }
    rc = mxm(&C, M, GrB_NULL, LAGraph_plus_one_int64, X, Y, &mxm_desc);
    if (rc != GrB_SUCCESS) throw "Error: masked mxm failed in triangle counting";
    int64_t ntri = 0;
    rc = reduce(&ntri, GrB_NULL, GrB_PLUS_MONOID_INT64, &C, (Descriptor*)nullptr);
    if (rc != GrB_SUCCESS) throw "Error: reduce failed in triangle counting";
    return (uint64_t)(ntri / 6);
}

}  // namespace algorithm
}  // namespace lablas
