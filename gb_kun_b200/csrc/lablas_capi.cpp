// libgbk_lablas.so: C entry points for the algorithms written against the
// lablas:: C++ API (host C++, no device code: everything on the GPU goes
// through libgbk.so).
#include <chrono>
#include <cstring>
#include <memory>
#include <string>

#include "lablas/gb_kun.h"
#include "algorithms/bfs.hpp"
#include "algorithms/cc.hpp"
#include "algorithms/pr.hpp"
#include "algorithms/sssp.hpp"
#include "algorithms/tc.hpp"
#include "gbk_lablas.h"

namespace {

thread_local std::string g_err;

struct Graph {
    int64_t n = 0;
    std::vector<int32_t> rp, col, w;
    std::unique_ptr<lablas::Matrix<float>> Af;  // unit values
    std::unique_ptr<lablas::Matrix<int>> Ai;    // unit values
    std::unique_ptr<lablas::Matrix<float>> Wf;  // weights as float
    std::unique_ptr<lablas::Matrix<int>> Wi;    // int32 weights
    std::unique_ptr<lablas::Matrix<float>> S;   // spmv values

    template <typename T>
    std::unique_ptr<lablas::Matrix<T>> make(const std::vector<T>& vals) {
        auto m = std::make_unique<lablas::Matrix<T>>();
        m->build_from_csr_arrays32(rp.data(), col.data(), vals.data(), n, (Index)col.size());
        return m;
    }
    lablas::Matrix<float>* unit_f() {
        if (!Af) Af = make<float>(std::vector<float>(col.size(), 1.0f));
        return Af.get();
    }
    // The unit matrix with the storage format the autotuner picks for its
    // unmasked plus-second SpMV (PageRank's product), tuned once per graph;
    // masked and sparse products keep using the CSR / CSC views.
    bool tuned_pr = false;
    lablas::Matrix<float>* pagerank_matrix() {
        auto* A = unit_f();
        if (!tuned_pr) {
            gbk_tune_result r;
            lablas::throw_if(gbk_matrix_autotune(A->handle(), 0, GBK_PLUS_SECOND, 10, &r, lablas::stream()),
                             "PageRank format autotune");
            tuned_pr = true;
        }
        return A;
    }
    lablas::Matrix<int>* unit_i() {
        if (!Ai) Ai = make<int>(std::vector<int>(col.size(), 1));
        return Ai.get();
    }
    lablas::Matrix<float>* weights_f() {
        if (!Wf) Wf = w.empty() ? make<float>(std::vector<float>(col.size(), 1.0f))
                                : make<float>(std::vector<float>(w.begin(), w.end()));
        return Wf.get();
    }
    lablas::Matrix<int>* weights_i() {
        if (!Wi) Wi = w.empty() ? make<int>(std::vector<int>(col.size(), 1)) : make<int>(std::vector<int>(w.begin(), w.end()));
        return Wi.get();
    }
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Timer {
    double* out;
    double t0;
    explicit Timer(double* o) : out(o) {
        cudaDeviceSynchronize();
        t0 = now_ms();
    }
    void stop() {
        cudaDeviceSynchronize();
        if (out) *out = now_ms() - t0;
    }
};

template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const char* e) {
        g_err = e;
        return GBK_PANIC;
    } catch (const std::exception& e) {
        g_err = e.what();
        return GBK_PANIC;
    }
}

template <typename T, typename O>
void copy_out(lablas::Vector<T>& v, O* out) {
    const T* h = v.host_dense();
    for (Index i = 0; i < v.size(); i++) out[i] = (O)h[i];
}

}  // namespace

struct gbk_lablas_graph_s : Graph {};

extern "C" {

int gbk_lablas_get_last_error(char* buf, size_t len) {
    if (!buf || !len) return GBK_NULL_POINTER;
    std::strncpy(buf, g_err.c_str(), len - 1);
    buf[len - 1] = 0;
    return 0;
}

int gbk_lablas_graph_create(gbk_lablas_graph* out, int64_t n, const int32_t* row_ptr, const int32_t* col,
                            const int32_t* weights) {
    if (!out || !row_ptr || (row_ptr[n] > 0 && !col)) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* g = new gbk_lablas_graph_s();
        g->n = n;
        g->rp.assign(row_ptr, row_ptr + n + 1);
        g->col.assign(col, col + row_ptr[n]);
        if (weights) g->w.assign(weights, weights + row_ptr[n]);
        *out = g;
        return 0;
    });
}

int gbk_lablas_graph_from_file(gbk_lablas_graph* out, const char* path) {
    if (!out || !path) return GBK_NULL_POINTER;
    return guarded([&] {
        auto m = std::make_unique<lablas::Matrix<float>>();
        m->init_from_mtx(path);
        if (m->ncols() != m->nrows()) throw "graph file: the algorithms need a square matrix (rows == cols)";
        auto* g = new gbk_lablas_graph_s();
        g->n = m->nrows();
        g->rp = m->host_row_ptr();
        g->col = m->host_col();
        g->Af = std::move(m);
        *out = g;
        return 0;
    });
}

int gbk_lablas_graph_destroy(gbk_lablas_graph g) {
    delete g;
    return 0;
}

int gbk_lablas_bfs(gbk_lablas_graph g, int64_t source, int32_t* levels, double* ms) {
    if (!g || !levels) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->unit_f();
        lablas::Vector<float> lv(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        lablas::algorithm::bfs_blast(&lv, A, (Index)source, &desc);
        t.stop();
        copy_out(lv, levels);
        return 0;
    });
}

int gbk_lablas_bfs_ops(gbk_lablas_graph g, int64_t source, int32_t* levels, double* ms) {
    if (!g || !levels) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->unit_f();
        lablas::Vector<float> lv(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        lablas::algorithm::bfs_blast_ops(&lv, A, (Index)source, &desc);
        t.stop();
        copy_out(lv, levels);
        return 0;
    });
}

int gbk_lablas_cc(gbk_lablas_graph g, int32_t* labels, int32_t* iterations, double* ms) {
    if (!g || !labels) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->unit_i();
        lablas::Vector<int> comp(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        Index it = lablas::algorithm::cc(&comp, A, 0, &desc);
        t.stop();
        if (iterations) *iterations = (int32_t)it;
        copy_out(comp, labels);
        return 0;
    });
}

int gbk_lablas_cc_fastsv(gbk_lablas_graph g, int32_t* labels, int32_t* iterations, double* ms) {
    if (!g || !labels) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->unit_i();
        lablas::Vector<int> comp(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        Index it = lablas::algorithm::cc_fastsv(&comp, A, 0, &desc);
        t.stop();
        if (iterations) *iterations = (int32_t)it;
        copy_out(comp, labels);
        return 0;
    });
}

int gbk_lablas_sssp_f32(gbk_lablas_graph g, int64_t source, float* dist, double* ms) {
    if (!g || !dist) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->weights_f();
        lablas::Vector<float> d(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        lablas::algorithm::sssp_bellman_ford_blast(&d, A, (Index)source, &desc);
        t.stop();
        copy_out(d, dist);
        return 0;
    });
}

int gbk_lablas_sssp_f32_ops(gbk_lablas_graph g, int64_t source, float* dist, double* ms) {
    if (!g || !dist) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->weights_f();
        lablas::Vector<float> d(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        lablas::algorithm::sssp_bellman_ford_blast_ops(&d, A, (Index)source, &desc);
        t.stop();
        copy_out(d, dist);
        return 0;
    });
}

int gbk_lablas_sssp_i32(gbk_lablas_graph g, int64_t source, int32_t* dist, double* ms) {
    if (!g || !dist) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->weights_i();
        lablas::Vector<int> d(g->n);
        lablas::Descriptor desc;
        Timer t(ms);
        lablas::algorithm::sssp_bellman_ford_blast(&d, A, (Index)source, &desc);
        t.stop();
        copy_out(d, dist);
        return 0;
    });
}

int gbk_lablas_pagerank(gbk_lablas_graph g, int32_t itermax, double damping, double tol, float* ranks,
                        int32_t* iterations, double* ms) {
    if (!g || !ranks) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->pagerank_matrix();
        LAGraph_Graph<float> graph(*A);
        lablas::Vector<float> r(g->n);
        int iters = 0;
        Timer t(ms);
        lablas::algorithm::page_rank_sinks(&r, &graph, &iters, itermax, damping, tol);
        t.stop();
        if (iterations) *iterations = iters;
        copy_out(r, ranks);
        return 0;
    });
}

int gbk_lablas_pagerank_ops(gbk_lablas_graph g, int32_t itermax, double damping, double tol, float* ranks,
                        int32_t* iterations, double* ms) {
    if (!g || !ranks) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->pagerank_matrix();
        LAGraph_Graph<float> graph(*A);
        lablas::Vector<float> r(g->n);
        int iters = 0;
        Timer t(ms);
        lablas::algorithm::page_rank_sinks_ops(&r, &graph, &iters, itermax, damping, tol);
        t.stop();
        if (iterations) *iterations = iters;
        copy_out(r, ranks);
        return 0;
    });
}

int gbk_lablas_ppr(gbk_lablas_graph g, int64_t seed, int32_t itermax, double damping, double tol, float* ranks,
                   int32_t* iterations, double* ms) {
    if (!g || !ranks) return GBK_NULL_POINTER;
    if (seed < 0 || seed >= g->n) return GBK_INVALID_INDEX;
    return guarded([&] {
        auto* A = g->pagerank_matrix();
        LAGraph_Graph<float> graph(*A);
        lablas::Vector<float> r(g->n);
        int iters = 0;
        Timer t(ms);
        lablas::algorithm::personalized_page_rank(&r, &graph, (Index)seed, &iters, itermax, damping, tol);
        t.stop();
        if (iterations) *iterations = iters;
        copy_out(r, ranks);
        return 0;
    });
}

int gbk_lablas_tc_method(gbk_lablas_graph g, int32_t method, uint64_t* count, double* ms) {
    if (!g || !count) return GBK_NULL_POINTER;
    if (method < 0 || method > 6) return GBK_INVALID_VALUE;
    return guarded([&] {
        auto* A = g->unit_i();
        Timer t(ms);
        *count = lablas::algorithm::triangle_count(A, method);
        t.stop();
        return 0;
    });
}

int gbk_lablas_tc(gbk_lablas_graph g, uint64_t* count, double* ms) {
    if (!g || !count) return GBK_NULL_POINTER;
    return guarded([&] {
        auto* A = g->unit_i();
        Timer t(ms);
        *count = lablas::algorithm::triangle_count_burkhardt(A);
        t.stop();
        return 0;
    });
}

int gbk_lablas_spmv(gbk_lablas_graph g, int32_t format, const float* vals, const float* x, float* y, double* ms) {
    if (!g || !vals || !x || !y) return GBK_NULL_POINTER;
    return guarded([&] {
        std::vector<float> v(vals, vals + g->col.size());
        auto A = g->make<float>(v);
        A->set_preferred_matrix_format((MatrixStorageFormat)format);
        lablas::Vector<float> u(g->n), w(g->n);
        u.build(x, g->n);
        w.fill(1.0f);
        lablas::Descriptor desc;
        Timer t(ms);
        lablas::mxv(&w, (lablas::Vector<float>*)nullptr, GrB_NULL, lablas::PlusMultipliesSemiring<float>(), A.get(),
                    &u, &desc);
        t.stop();
        copy_out(w, y);
        return 0;
    });
}

}  // extern "C"
