// PageRank through the lablas:: API, following LAGraph's page_rank_sinks as
// the reference ports it (algorithms/pr/pr.hpp:20-153): graph AT = A,
// d_out = column degrees, d = max(d_out / damping, 1 / damping), sinks (zero
// column degree) redistribute their rank through the teleport term, and each
// iteration computes r = teleport + A (t ./ d) with a plus-second mxv.
// Unlike the reference, which always runs itermax iterations, the loop stops
// once rdiff < tol when tol > 0 (the stopping rule LAGraph documents); with
// tol <= 0 it runs exactly itermax iterations like the reference.
//
//  * page_rank_sinks runs the loop on the device (gbk_pagerank: the SpMV in
//    the matrix's format, one fused element-wise pass, a control kernel; one
//    CUDA graph for the iterations).
//  * page_rank_sinks_ops is the same iteration as the reference's sequence
//    of GraphBLAS calls, with a host read of rdiff per iteration.
#pragma once

#include "lablas/gb_kun.h"

namespace lablas {
namespace algorithm {

inline void page_rank_sinks(Vector<float>* centrality, LAGraph_Graph<float>* G, int* iters, int itermax = 100,
                            double damping = 0.85, double tol = 1e-4) {
    int32_t it = 0;
    throw_if(gbk_pagerank(G->AT->handle(), itermax, damping, tol, centrality->dense_ptr(), &it, nullptr, stream()),
             "page_rank_sinks");
    *iters = it;
}

inline void page_rank_sinks_ops(Vector<float>* centrality, LAGraph_Graph<float>* G, int* iters, int itermax = 100,
                                double damping = 0.85, double tol = 1e-4) {
    Matrix<float>* AT = G->AT;
    Vector<Index>* d_out = G->coldegree;
    Descriptor desc;
    const Index n = AT->nrows();
    const float* none = nullptr;
    (void)none;
    const Vector<float>* NOMASK = nullptr;

    const double scaled_damping = (1 - damping) / n;
    float rdiff = 1;

    Vector<float> t(n), r(n), w(n), d(n), d1(n);
    Vector<float>* tp = &t;
    Vector<float>* rp = &r;

    assign(rp, NOMASK, GrB_NULL, 1.0 / n, GrB_ALL, n, (Descriptor*)nullptr);

    // sinks: zero column degree, found with a complemented structural mask
    Index nvals = 0;
    d_out->get_nvals(&nvals);
    const Index nsinks = n - nvals;
    Vector<bool> sink(n);
    Vector<float> rsink(n);
    if (nsinks > 0) assign(&sink, d_out, GrB_NULL, (bool)true, GrB_ALL, n, GrB_DESC_SC);

    // d = max(d_out / damping, 1 / damping)
    apply(&d, NOMASK, GrB_NULL, GrB_DIV_FP32, d_out, damping, &desc);
    assign(&d1, NOMASK, GrB_NULL, (float)(1.0 / damping), GrB_ALL, n, (Descriptor*)nullptr);
    eWiseAdd(&d, NOMASK, GrB_NULL, GrB_MAX_FP32, &d1, &d, (Descriptor*)nullptr);

    for ((*iters) = 0; (*iters) < itermax; (*iters)++) {
        if (tol > 0 && rdiff < tol) break;
        float teleport = (float)scaled_damping;
        if (nsinks > 0) {
            const float damping_over_n = (float)(damping / n);
            rsink.clear();
            assign(&rsink, &sink, GrB_NULL, rp, GrB_ALL, n, GrB_DESC_S);
            float sum_rsink = 0;
            reduce(&sum_rsink, GrB_NULL, GrB_PLUS_MONOID_FP32, &rsink, (Descriptor*)nullptr);
            teleport += damping_over_n * sum_rsink;
        }
        std::swap(tp, rp);  // t is the old score
        eWiseMult(&w, NOMASK, GrB_NULL, GrB_DIV_FP32, tp, &d, (Descriptor*)nullptr);
        assign(rp, NOMASK, GrB_NULL, teleport, GrB_ALL, n, (Descriptor*)nullptr);
        mxv(rp, NOMASK, GrB_PLUS_FP32, LAGraph_plus_second_fp32, AT, &w, &desc);
        assign(tp, NOMASK, GrB_MINUS_FP32, rp, GrB_ALL, n, (Descriptor*)nullptr);
        apply(tp, NOMASK, GrB_NULL, GrB_ABS_FP32, tp, (Descriptor*)nullptr);
        rdiff = 0;
        reduce(&rdiff, GrB_NULL, GrB_PLUS_MONOID_FP32, tp, (Descriptor*)nullptr);
    }
    centrality->dup(rp);
}

// Personalised PageRank from one seed, built from the same lablas:: steps as
// page_rank_sinks (one plus-second mxv per iteration): r0 = e_seed and the
// teleport and sink mass return to the seed,
//   r = [(1 - damping) + damping * sum_{sinks} r] e_seed + A (r ./ d),
// stopping once sum |r_new - r| < tol (tol > 0) or after itermax iterations.
// The sink mass is a plain sum over the zero-column-degree vertices (dense
// vectors), not the reference's sparse-mask form.
inline void personalized_page_rank(Vector<float>* centrality, LAGraph_Graph<float>* G, Index seed, int* iters,
                                   int itermax = 100, double damping = 0.85, double tol = 1e-6) {
    Matrix<float>* AT = G->AT;
    Vector<Index>* d_out = G->coldegree;
    Descriptor desc;
    const Index n = AT->nrows();
    const Vector<float>* NOMASK = nullptr;
    float rdiff = 1;

    Vector<float> t(n), r(n), w(n), d(n), d1(n), sinkf(n), tmp(n), tv(n);
    Vector<float>* tp = &t;
    Vector<float>* rp = &r;
    assign(rp, NOMASK, GrB_NULL, 0.0f, GrB_ALL, n, (Descriptor*)nullptr);
    rp->set_element(1.0f, seed);
    assign(&tv, NOMASK, GrB_NULL, 0.0f, GrB_ALL, n, (Descriptor*)nullptr);
    // 1.0 where the column degree is zero (complemented structural mask)
    assign(&sinkf, NOMASK, GrB_NULL, 0.0f, GrB_ALL, n, (Descriptor*)nullptr);
    assign(&sinkf, d_out, GrB_NULL, 1.0f, GrB_ALL, n, GrB_DESC_SC);
    // d = max(d_out / damping, 1 / damping)
    apply(&d, NOMASK, GrB_NULL, GrB_DIV_FP32, d_out, damping, &desc);
    assign(&d1, NOMASK, GrB_NULL, (float)(1.0 / damping), GrB_ALL, n, (Descriptor*)nullptr);
    eWiseAdd(&d, NOMASK, GrB_NULL, GrB_MAX_FP32, &d1, &d, (Descriptor*)nullptr);

    for ((*iters) = 0; (*iters) < itermax; (*iters)++) {
        if (tol > 0 && rdiff < tol) break;
        eWiseMult(&tmp, NOMASK, GrB_NULL, multiplies<float>(), rp, &sinkf, (Descriptor*)nullptr);
        float sink = 0;
        reduce(&sink, GrB_NULL, GrB_PLUS_MONOID_FP32, &tmp, (Descriptor*)nullptr);
        const float teleport = (float)((1.0 - damping) + damping * sink);
        std::swap(tp, rp);  // t is the old score
        eWiseMult(&w, NOMASK, GrB_NULL, GrB_DIV_FP32, tp, &d, (Descriptor*)nullptr);
        assign(rp, NOMASK, GrB_NULL, 0.0f, GrB_ALL, n, (Descriptor*)nullptr);
        mxv(rp, NOMASK, GrB_PLUS_FP32, LAGraph_plus_second_fp32, AT, &w, &desc);
        tv.set_element(teleport, seed);
        eWiseAdd(rp, NOMASK, GrB_NULL, GrB_PLUS_FP32, rp, &tv, (Descriptor*)nullptr);
        assign(tp, NOMASK, GrB_MINUS_FP32, rp, GrB_ALL, n, (Descriptor*)nullptr);
        apply(tp, NOMASK, GrB_NULL, GrB_ABS_FP32, tp, (Descriptor*)nullptr);
        rdiff = 0;
        reduce(&rdiff, GrB_NULL, GrB_PLUS_MONOID_FP32, tp, (Descriptor*)nullptr);
    }
    centrality->dup(rp);
}

}  // namespace algorithm
}  // namespace lablas

// The LAGraph-named entry point of the reference (pr.hpp:20-27).
inline void LAGraph_page_rank_sinks(lablas::Vector<float>* centrality, LAGraph_Graph<float>* G, int* iters,
                                    int itermax = 100, double damping = 0.85, double tol = 1e-4) {
    // The reference never applies tol; keep that for the drop-in name.
    (void)tol;
    lablas::algorithm::page_rank_sinks(centrality, G, iters, itermax, damping, 0.0);
}
