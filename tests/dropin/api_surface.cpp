// Compile-only check of the drop-in header's surface (no GPU needed): the
// calls the reference's algorithm files and drivers make, with the element
// types they use, must compile against gb_kun_b200/dropin/src/gb_kun.h.
#include "src/gb_kun.h"

#define MASK_NULL static_cast<const lablas::Vector<float>*>(NULL)

void surface(lablas::Matrix<int>& A, lablas::Matrix<float>& F, Index n) {
    lablas::Descriptor desc;
    // vxm with a bool frontier over an int matrix and an int mask (bfs.hpp:60-70)
    lablas::Vector<bool>* frontier = nullptr;
    lablas::Vector<int>* level = nullptr;
    GrB_Vector_new(&frontier, GrB_BOOL, n);
    GrB_Vector_new(&level, GrB_INT32, n);
    GrB_Vector_setElement(frontier, true, 0);
    frontier->print();
    GrB_assign(level, frontier, NULL, (Index)1, GrB_ALL, n, GrB_DESC_S);
    GrB_vxm(frontier, level, NULL, lablas::LogicalOrAndSemiring<bool>(), frontier, &A, GrB_DESC_RSC);
    Index nv = 0;
    GrB_Vector_nvals(&nv, frontier);
    // host CSR view and writable host copies (the *_traditional.hpp checkers)
    const lablas::backend::MatrixCSR<float>* csr = F.get_matrix()->get_csr();
    lablas::Vector<float> out(n);
    float* h = out.get_vector()->getDense()->get_vals();
    h[0] = (float)csr->get_row_ptr()[1] + (float)csr->get_col_ids()[0] + csr->get_vals()[0];
    lablas::Vector<bool> b(n);
    bool* hb = b.get_vector()->getDense()->get_vals();
    hb[0] = true;
    // statistics macros (stats.h:11-117)
    SAVE_STATS((GrB_TRY(GrB_mxv(&out, MASK_NULL, GrB_PLUS_FP32, LAGraph_plus_second_fp32, &F, &out, &desc))),
               "pr_mxv", (sizeof(float) * 2 + sizeof(size_t)), 1, &F);
    SAVE_TEPS((void)0, "noop", 1, &F);
    save_teps("noop", 1.0, 10, 1);
    // a select with a lambda compiles (and refuses to run on the device)
    auto tril = [](int x, Index i, Index j, int val) { return (j <= (i + val)) ? 0 : x; };
    lablas::Matrix<int> L;
    GrB_select(&L, static_cast<const lablas::Matrix<float>*>(NULL), NULL, tril, &A, (int64_t)-1, NULL);
    GrB_free(&frontier);
    GrB_free(&level);
}
