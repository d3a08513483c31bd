// Connected components through the lablas:: API with the result of the
// FastSV loop of algorithms/cc/cc.hpp:12-119 (Zhang, Azad and Hu, SIAM PP20):
// every vertex labelled with the smallest vertex id of its component.
//
//  * cc_fastsv is that loop as the reference writes it: stochastic hooking
//    through the minimum grandparent among neighbours (min-select-second
//    mxv), aggressive hooking and shortcutting with min eWiseAdds,
//    grandparents by extract, termination when no grandparent changes (a
//    host read per iteration).
//  * cc reaches the same labels on a symmetric matrix with a lock-free
//    union-find on the device (gbk_cc_labels, three launches, no host round
//    trip) and runs cc_fastsv on any other matrix, where FastSV's fixed
//    point need not be the weakly connected components.
#pragma once

#include <limits>

#include "lablas/gb_kun.h"

namespace lablas {
namespace algorithm {

inline Index cc_fastsv(Vector<int>* v, const Matrix<int>* A, int seed, Descriptor* desc) {
    (void)seed;
    // The reference builds CC with __DISABLE_SPMSPV__ (cc.cpp:2): the hooking
    // mxv always reads the grandparent vector densely, zeros included.
    ScopedDisableSpMSpV dense_mxv;
    Index n;
    A->get_nrows(&n);
    const Vector<int>* NOMASK = nullptr;
    Vector<bool> diff(n);
    Vector<int> parent(n), parent_temp(n);
    Vector<int> grandparent(n), grandparent_temp(n);
    Vector<int> mngp(n), mngp_temp(n);

    parent.fillAscending(n);
    mngp.dup(&parent);
    mngp_temp.dup(&parent);
    grandparent.dup(&parent);
    grandparent_temp.dup(&parent);

    Index succ = 0;
    const Index niter = 100;
    Index iter;
    for (iter = 1; iter <= niter; ++iter) {
        parent_temp.dup(&parent);
        // 1) stochastic hooking: mngf = A min.second gf, then f[f[u]] = mngf[u]
        mxv(&mngp_temp, NOMASK, GrB_NULL, MinimumSelectSecondSemiring<int>(), A, &grandparent, desc);
        eWiseAdd(&mngp, NOMASK, GrB_NULL, MinimumSelectSecondSemiring<int>(), &mngp, &mngp_temp, desc);
        assignScatter(&parent, NOMASK, GrB_NULL, &mngp, &parent_temp, parent_temp.nvals(), desc);
        // 2) aggressive hooking: f = min(f, mngf)
        eWiseAdd(&parent, NOMASK, GrB_NULL, MinimumPlusSemiring<int>(), &parent, &mngp, desc);
        // 3) shortcutting: f = min(f, old f)
        eWiseAdd(&parent, NOMASK, GrB_NULL, MinimumPlusSemiring<int>(), &parent, &parent_temp, desc);
        // 4) grandparents: gf[u] = f[f[u]]
        extract(&grandparent, NOMASK, GrB_NULL, &parent, &parent, desc);
        // 5) termination: no grandparent changed
        eWiseMult(&diff, NOMASK, GrB_NULL, MinimumNotEqualToSemiring<int, int, bool>(), &grandparent_temp,
                  &grandparent, desc);
        succ = 0;
        reduce<Index, bool>(&succ, GrB_NULL, PlusMonoid<Index>(), &diff, desc);
        if (succ == 0) break;
        grandparent_temp.dup(&grandparent);
        // 6) deactivate unchanged vertices (under the toggled descriptor, as the reference does)
        desc->toggle(GrB_MASK);
        assign(&grandparent, &diff, nullptr, std::numeric_limits<int>::max(), GrB_ALL, n, desc);
        desc->toggle(GrB_MASK);
    }
    v->dup(&parent);
    return iter;
}

// Returns FastSV's iteration count, or 0 when the union-find labelled A.
inline Index cc(Vector<int>* v, const Matrix<int>* A, int seed, Descriptor* desc) {
    int32_t symmetric = 0;
    throw_if(gbk_matrix_pattern_symmetric(A->handle(), &symmetric, stream()), "cc");
    if (!symmetric) return cc_fastsv(v, A, seed, desc);
    throw_if(gbk_cc_labels(A->handle(), GBK_I32, v->dense_ptr(), stream()), "cc");
    return 0;
}

}  // namespace algorithm
}  // namespace lablas
