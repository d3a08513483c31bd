// Bellman-Ford SSSP through the lablas:: API with the distances of
// algorithms/sssp/sssp_blast.hpp:8-72: distances start at the type's maximum
// ("infinity") with 0 at the source; T = float restates the reference exactly
// (integer weights below 2^24 are exact in float); T = int runs with int32
// weights and saturating additions.
//
//  * sssp_bellman_ford_blast runs a label-correcting near-far worklist on the
//    device (gbk_sssp_dist, one graph launch for all rounds).  Each distance is the
//    minimum over walks of the left-to-right rounded sums either way, since
//    rounding is monotone, so the result equals the reference's.
//  * sssp_bellman_ford_blast_ops is the reference's own sequence: every
//    round relaxes all edges out of the current frontier vector with a
//    min-plus vxm, records which vertices improved (custom-less eWiseAdd),
//    keeps the minimum and stops when no vertex improves (a host read per
//    round).
#pragma once

#include <limits>

#include "lablas/gb_kun.h"

namespace lablas {
namespace algorithm {

// Returns the worklist rounds run.
template <typename T>
Index sssp_bellman_ford_blast(Vector<T>* v, const Matrix<T>* A, Index s, Descriptor* desc) {
    (void)desc;
    int32_t rounds = 0;
    throw_if(gbk_sssp_dist(A->handle(), (int64_t)s, 0.0, v->dense_ptr(), &rounds, stream()),
             "sssp_bellman_ford_blast");
    return rounds;
}

template <typename T>
Index sssp_bellman_ford_blast_ops(Vector<T>* v, const Matrix<T>* A, Index s, Descriptor* desc) {
    const Index n = A->nrows();
    const T inf = std::numeric_limits<T>::max();
    v->fill(inf);
    v->set_element((T)0, s);
    Vector<T> f1(n);
    Vector<T> f2(n);
    f1.fill(inf);
    f1.set_element((T)0, s);
    Vector<T> m(n);

    Index iter;
    Index f1_nvals = 1;
    T succ = 1;
    for (iter = 1; iter <= n; ++iter) {
        vxm<T, T, T, T>(&f2, nullptr, GrB_NULL, MinimumPlusSemiring<T>(), &f1, A, desc);
        eWiseAdd<T, T, T, T>(&m, nullptr, GrB_NULL, CustomLessPlusSemiring<T>(), &f2, v, desc);
        eWiseAdd<T, T, T, T>(v, nullptr, GrB_NULL, MinimumPlusSemiring<T>(), v, &f2, desc);
        // As in the reference, the toggled descriptor holds GrB_SCMP here,
        // a mode the masked assign leaves untouched.
        desc->toggle(GrB_MASK);
        assign<T, T, T>(&f2, &m, GrB_NULL, inf, GrB_ALL, n, desc);
        desc->toggle(GrB_MASK);
        f2.swap(&f1);
        f1_nvals = f1.nvals();
        succ = 0;
        reduce<T, T>(&succ, GrB_NULL, PlusMonoid<T>(), &m, desc);
        if (f1_nvals == 0 || succ == 0) break;
    }
    return iter;
}

}  // namespace algorithm
}  // namespace lablas
