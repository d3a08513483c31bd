// Triangle counting, Burkhardt's method (algorithms/tc/tc.hpp:88-284, the
// default of LAGr_TriangleCount): C<A> = A (+.one) A counts, for every edge
// (i, j), the common neighbours of i and j; sum(C) / 6 is the number of
// triangles of the symmetric graph A.
#pragma once

#include <cstdint>

#include "lablas/gb_kun.h"

namespace lablas {
namespace algorithm {

inline uint64_t triangle_count_burkhardt(const Matrix<int>* A) {
    Matrix<int> C;
    Descriptor mxm_desc({{GrB_MXMMODE, GrB_IKJ_MASKED}});
    LA_Info rc = mxm(&C, A, GrB_NULL, LAGraph_plus_one_int64, A, A, &mxm_desc);
    if (rc != GrB_SUCCESS) throw "Error: masked mxm failed in triangle counting";
    int64_t ntri = 0;
    rc = reduce(&ntri, GrB_NULL, GrB_PLUS_MONOID_INT64, &C, (Descriptor*)nullptr);
    if (rc != GrB_SUCCESS) throw "Error: reduce failed in triangle counting";
    return (uint64_t)(ntri / 6);
}

}  // namespace algorithm
}  // namespace lablas
