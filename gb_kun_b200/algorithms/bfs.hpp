// Level-synchronous BFS through the lablas:: API with the result of the
// GraphBLAST "blast" formulation of algorithms/bfs/bfs.hpp:94-142: levels
// start at 1 for the source, 0 marks unvisited, edges are followed along the
// rows of A.
//
//  * bfs_blast runs the whole level loop on the device (gbk_bfs_levels:
//    direction-optimising, one CUDA graph launch per search).
//  * bfs_blast_ops is the reference's own sequence of GraphBLAS calls: each
//    level assigns the frontier's level, then expands the frontier with an
//    or-and vxm masked by the complement of the visited set (a sparse
//    frontier pushed through SpMSpV over the CSR, a dense one pulled through
//    a masked SpMV over the CSC, as backend::vxm decides) and reads the
//    frontier's size back to the host.
#pragma once

#include "lablas/gb_kun.h"

namespace lablas {
namespace algorithm {

template <typename T>
void bfs_blast(Vector<T>* v, const Matrix<T>* A, Index s, Descriptor* desc) {
    (void)desc;
    throw_if(gbk_bfs_levels(A->handle(), (int64_t)s, 0, Vector<T>::dtype, v->dense_ptr(), nullptr, stream()),
             "bfs_blast");
}

template <typename T>
void bfs_blast_ops(Vector<T>* v, const Matrix<T>* A, Index s, Descriptor* desc) {
    const Index n = A->nrows();
    v->fill((T)0);
    Vector<T> f1(n);
    Vector<T> f2(n);
    f1.fill((T)0);
    f1.set_element((T)1, s);

    T succ = 0;
    for (Index iter = 1; iter <= n; ++iter) {
        assign<T, T, T>(v, &f1, GrB_NULL, (T)iter, GrB_ALL, n, desc);
        desc->toggle(GrB_MASK);
        vxm<T, T, T, T>(&f2, v, GrB_NULL, LogicalOrAndSemiring<T>(), &f1, A, GrB_DESC_SC);
        desc->toggle(GrB_MASK);
        f2.swap(&f1);
        succ = 0;
        reduce<T, T>(&succ, GrB_NULL, PlusMonoid<T>(), &f1, desc);
        if (succ == 0) break;
    }
}

}  // namespace algorithm
}  // namespace lablas
