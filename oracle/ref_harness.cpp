// Harness around the reference library's own CPU code (GB_Kun, header-only
// C++ with OpenMP).  TEST INFRASTRUCTURE ONLY: built by oracle/Makefile from
// the reference sources where they lie into oracle/_ref/ (git-ignored), and
// loaded only by tests/, tests/golden/make_golden.py and bench.py's
// reference / cpu_baseline legs.
//
// This is the one translation unit that includes the reference's gb_kun.h
// (it defines non-inline functions, so it can be included once per binary).
// Inputs are the build's int32 CSR arrays, widened to the reference's
// 64-bit Index and passed to lablas::Matrix<T>::build_from_csr_arrays
// (src/cpp_graphblas/matrix.hpp:93-105).  Each entry point times only the
// reference call (std::chrono::steady_clock, median of `reps` after `warmup`).
//
// Built twice: once as is, once with __DISABLE_SPMSPV__ (the switch cc.cpp:2
// sets for connected components).

#include "src/gb_kun.h"
#include "algorithms/bfs/bfs.hpp"
#include "algorithms/pr/pr.hpp"
#include "algorithms/cc/cc.hpp"
#include "algorithms/sssp/sssp_blast.hpp"
#include "algorithms/tc/tc.hpp"

#include <chrono>
#include <cstdint>
#include <streambuf>
#include <vector>

namespace {

struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};

struct Quiet {  // silence the reference's progress printing during a call
    NullBuf nb;
    std::streambuf* old;
    Quiet() : old(std::cout.rdbuf(&nb)) {}
    ~Quiet() { std::cout.rdbuf(old); }
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

double median(std::vector<double> v) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    size_t m = v.size() / 2;
    return (v.size() % 2) ? v[m] : 0.5 * (v[m - 1] + v[m]);
}

template <typename T>
void build(lablas::Matrix<T>& A, int format, int64_t n, const int32_t* rp, const int32_t* col, const T* val) {
    int64_t nnz = rp[n];
    std::vector<Index> rp64(rp, rp + n + 1), col64(col, col + nnz);
    std::vector<T> v(val, val + nnz);
    A.set_preferred_matrix_format((MatrixStorageFormat)format);
    A.build_from_csr_arrays(rp64.data(), col64.data(), v.data(), (Index)n, (Index)nnz);
}

}  // namespace

extern "C" {

int ref_max_threads() { return omp_get_max_threads(); }

// y = A x with the reference's GrB_mxv (spmv.cpp:83-92) in the chosen
// storage format.  semiring: 0 plus-times, 1 or-and, 6 min-plus,
// 8 min-select-second, 4 plus-second (gbk_semiring values).
int ref_spmv(int format, int semiring, int64_t n, const int32_t* rp, const int32_t* col, const float* val,
             const float* x, float* y, int warmup, int reps, double* ms_median) {
    try {
        Quiet q;
        lablas::Matrix<float> A;
        build(A, format, n, rp, col, val);
        lablas::Vector<float> u(n), w(n);
        u.build(x, n);
        lablas::Descriptor desc;
        std::vector<double> times;
        for (int r = 0; r < warmup + reps; r++) {
            w.fill(1.0f);
            double t0 = now_ms();
            switch (semiring) {
                case 0: lablas::mxv(&w, (lablas::Vector<float>*)NULL, NULL, lablas::PlusMultipliesSemiring<float>(), &A, &u, &desc); break;
                case 1: lablas::mxv(&w, (lablas::Vector<float>*)NULL, NULL, lablas::LogicalOrAndSemiring<float>(), &A, &u, &desc); break;
                case 4: lablas::mxv(&w, (lablas::Vector<float>*)NULL, NULL, lablas::PlusSecondSemiring<float>(), &A, &u, &desc); break;
                case 6: lablas::mxv(&w, (lablas::Vector<float>*)NULL, NULL, lablas::MinimumPlusSemiring<float>(), &A, &u, &desc); break;
                case 8: lablas::mxv(&w, (lablas::Vector<float>*)NULL, NULL, lablas::MinimumSelectSecondSemiring<float>(), &A, &u, &desc); break;
                default: return 5;
            }
            double t1 = now_ms();
            if (r >= warmup) times.push_back(t1 - t0);
        }
        const float* out = w.get_vector()->getDense()->get_vals();
        std::copy(out, out + n, y);
        if (ms_median) *ms_median = median(times);
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// BFS levels (source = 1, unvisited = 0) from bfs_blast (algorithms/bfs/bfs.hpp:93-142).
int ref_bfs(int64_t n, const int32_t* rp, const int32_t* col, int32_t source, int32_t* levels, int reps,
            double* ms_median) {
    try {
        Quiet q;
        std::vector<float> ones(rp[n], 1.0f);
        lablas::Matrix<float> A;
        build(A, 0, n, rp, col, ones.data());
        lablas::Vector<float> lv(n);
        lablas::Descriptor desc;
        std::vector<double> times;
        for (int r = 0; r < (reps > 0 ? reps : 1); r++) {
            double t0 = now_ms();
            lablas::algorithm::bfs_blast(&lv, &A, (Index)source, &desc);
            times.push_back(now_ms() - t0);
        }
        const float* out = lv.get_vector()->getDense()->get_vals();
        for (int64_t i = 0; i < n; i++) levels[i] = (int32_t)out[i];
        if (ms_median) *ms_median = median(times);
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// Connected-component labels from FastSV cc (algorithms/cc/cc.hpp:12-119).
int ref_cc(int64_t n, const int32_t* rp, const int32_t* col, int32_t* labels, int reps, double* ms_median) {
    try {
        Quiet q;
        std::vector<int> ones(rp[n], 1);
        lablas::Matrix<int> A;
        build(A, 0, n, rp, col, ones.data());
        lablas::Vector<int> comp(n);
        lablas::Descriptor desc;
        std::vector<double> times;
        for (int r = 0; r < (reps > 0 ? reps : 1); r++) {
            double t0 = now_ms();
            lablas::algorithm::cc(&comp, &A, 0, &desc);
            times.push_back(now_ms() - t0);
        }
        const int* out = comp.get_vector()->getDense()->get_vals();
        for (int64_t i = 0; i < n; i++) labels[i] = out[i];
        if (ms_median) *ms_median = median(times);
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// SSSP distances from sssp_bellman_ford_blast (algorithms/sssp/sssp_blast.hpp:8-72),
// integer weights passed as exact floats; unreachable = FLT_MAX.
int ref_sssp(int64_t n, const int32_t* rp, const int32_t* col, const int32_t* w, int32_t source, float* dist,
             int reps, double* ms_median) {
    try {
        Quiet q;
        std::vector<float> wf(w, w + rp[n]);
        lablas::Matrix<float> A;
        build(A, 0, n, rp, col, wf.data());
        lablas::Vector<float> d(n);
        lablas::Descriptor desc;
        std::vector<double> times;
        for (int r = 0; r < (reps > 0 ? reps : 1); r++) {
            double t0 = now_ms();
            lablas::algorithm::sssp_bellman_ford_blast(&d, &A, (Index)source, &desc);
            times.push_back(now_ms() - t0);
        }
        const float* out = d.get_vector()->getDense()->get_vals();
        std::copy(out, out + n, dist);
        if (ms_median) *ms_median = median(times);
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// PageRank from LAGraph_page_rank_sinks (algorithms/pr/pr.hpp:20-153); runs
// exactly `iters` iterations (the reference does not stop on tol).
int ref_pr(int64_t n, const int32_t* rp, const int32_t* col, int iters, float* ranks, int reps,
           double* ms_median) {
    try {
        Quiet q;
        std::vector<float> ones(rp[n], 1.0f);
        lablas::Matrix<float> A;
        build(A, 0, n, rp, col, ones.data());
        LAGraph_Graph<float> graph(A);
        lablas::Vector<float> r(n);
        std::vector<double> times;
        for (int k = 0; k < (reps > 0 ? reps : 1); k++) {
            int taken = 0;
            double t0 = now_ms();
            LAGraph_page_rank_sinks(&r, &graph, &taken, iters);
            times.push_back(now_ms() - t0);
        }
        const float* out = r.get_vector()->getDense()->get_vals();
        std::copy(out, out + n, ranks);
        if (ms_median) *ms_median = median(times);
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// Triangle count, Burkhardt method with masked IKJ SpGEMM (algorithms/tc/tc.hpp:88-284).
int ref_tc(int64_t n, const int32_t* rp, const int32_t* col, uint64_t* count, int reps, double* ms_median) {
    try {
        Quiet q;
        std::vector<int> ones(rp[n], 1);
        lablas::Matrix<int> A;
        build(A, 0, n, rp, col, ones.data());
        LAGraph_Graph<int> graph(A);
        std::vector<double> times;
        uint64_t ntri = 0;
        for (int k = 0; k < (reps > 0 ? reps : 1); k++) {
            double t0 = now_ms();
            lablas::algorithm::LAGr_TriangleCount(&ntri, &graph, lablas::algorithm::LAGraph_TriangleCount_Burkhardt,
                                                  lablas::algorithm::LAGraph_TriangleCount_NoSort,
                                                  &lablas::GrB_DESC_IKJ_MASKED);
            times.push_back(now_ms() - t0);
        }
        *count = ntri;
        if (ms_median) *ms_median = median(times);
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// Graph file through the reference's own reader: lablas::Matrix<T>::
// init_from_mtx (src/cpp_graphblas/matrix.hpp:107-110 -> read_file.hpp:565-617)
// in the CSR storage format.  The matrix stays alive behind *handle until
// ref_graph_free; ref_graph_csr copies its CSR out (int32).  At least four
// OpenMP threads are used for .mtxbin (binary_read_mtx_file runs
// omp_get_max_threads() / 4 threads, read_file.hpp:428).
int ref_graph_read(const char* path, int64_t* nrows, int64_t* nnz, void** handle, double* ms) {
    try {
        Quiet q;
        const int before = omp_get_max_threads();
        if (before < 4) omp_set_num_threads(4);
        auto* A = new lablas::Matrix<float>();
        A->get_matrix()->set_preferred_matrix_format(CSR);
        const double t0 = now_ms();
        A->init_from_mtx(path);
        if (ms) *ms = now_ms() - t0;
        omp_set_num_threads(before);
        const lablas::backend::MatrixCSR<float>* csr = A->get_matrix()->get_csr();
        *nrows = (int64_t)A->get_matrix()->get_nrows();
        *nnz = (int64_t)csr->get_nnz();
        *handle = A;
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

int ref_graph_csr(void* handle, int32_t* rp, int32_t* col, float* val) {
    auto* A = (lablas::Matrix<float>*)handle;
    const lablas::backend::MatrixCSR<float>* csr = A->get_matrix()->get_csr();
    const int64_t n = (int64_t)A->get_matrix()->get_nrows(), nnz = (int64_t)csr->get_nnz();
    const ENT* p = csr->get_row_ptr();
    const VNT* c = csr->get_col_ids();
    const float* v = csr->get_vals();
    for (int64_t i = 0; i <= n; i++) rp[i] = (int32_t)p[i];
    for (int64_t e = 0; e < nnz; e++) {
        col[e] = (int32_t)c[e];
        if (val) val[e] = v[e];
    }
    return 0;
}

void ref_graph_free(void* handle) { delete (lablas::Matrix<float>*)handle; }

// Unmasked SpGEMM C = A (+.x) A through the reference's mxm with a NULL
// mask (src/backend/operations/operations.h:476-482 -> SpMSpM_unmasked_ikj,
// spmspm_hash_based_gustavson.h:9-148).  semiring (gbk_semiring values):
// 0 plus-times, 1 or-and, 6 min-plus, 10 plus-one.  C stays alive behind
// *handle (read it with ref_graph_csr, free it with ref_graph_free).
int ref_mxm(int semiring, int64_t n, const int32_t* rp, const int32_t* col, const float* val, void** handle,
            int64_t* nnz, double* ms) {
    try {
        Quiet q;
        lablas::Matrix<float> A;
        build(A, 0, n, rp, col, val);
        auto* C = new lablas::Matrix<float>();
        lablas::Descriptor desc;
        const lablas::Matrix<float>* nomask = nullptr;
        const auto acc = lablas::second<float, float, float>();
        LA_Info rc = GrB_SUCCESS;
        const double t0 = now_ms();
        switch (semiring) {
            case 0: rc = lablas::mxm(C, nomask, acc, lablas::PlusMultipliesSemiring<float>(), &A, &A, &desc); break;
            case 1: rc = lablas::mxm(C, nomask, acc, lablas::LogicalOrAndSemiring<float>(), &A, &A, &desc); break;
            case 6: rc = lablas::mxm(C, nomask, acc, lablas::MinimumPlusSemiring<float>(), &A, &A, &desc); break;
            case 10: rc = lablas::mxm(C, nomask, acc, lablas::PlusOneSemiring<float>(), &A, &A, &desc); break;
            default: delete C; return 5;
        }
        if (ms) *ms = now_ms() - t0;
        if (rc != GrB_SUCCESS) {
            delete C;
            return (int)rc;
        }
        *nnz = (int64_t)C->get_matrix()->get_csr()->get_nnz();
        *handle = C;
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// Matrix select through the reference's select (select.h:363-395) with an
// index-unary operator (gbk_select_op values): 0 tril, 1 triu, 2 diag,
// 3 offdiag (k = thunk), 4..9 value ==, !=, >, >=, <, <= thunk; the
// operator returns the value where it keeps the entry and 0 elsewhere.
int ref_select_matrix(int op, double thunk, int64_t n, const int32_t* rp, const int32_t* col, const float* val,
                      void** handle) {
    try {
        Quiet q;
        lablas::Matrix<float> U;
        build(U, 0, n, rp, col, val);
        auto* W = new lablas::Matrix<float>();
        const lablas::Matrix<float>* nomask = nullptr;
        lablas::Descriptor desc;
        const auto acc = lablas::second<float, float, float>();
        auto sel = [op](float x, Index i, Index j, double k) -> float {
            const Index ki = (Index)k;
            bool keep = false;
            switch (op) {
                case 0: keep = j <= i + ki; break;
                case 1: keep = j >= i + ki; break;
                case 2: keep = j == i + ki; break;
                case 3: keep = j != i + ki; break;
                case 4: keep = x == k; break;
                case 5: keep = x != k; break;
                case 6: keep = x > k; break;
                case 7: keep = x >= k; break;
                case 8: keep = x < k; break;
                case 9: keep = x <= k; break;
            }
            return keep ? x : 0.0f;
        };
        LA_Info rc = lablas::select(W, nomask, acc, sel, &U, thunk, &desc);
        if (rc != GrB_SUCCESS) {
            delete W;
            return (int)rc;
        }
        *handle = W;
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

// LAGr_TriangleCount with a method (algorithms/tc/tc.hpp:17-26), NoSort,
// masked IKJ SpGEMM as the default descriptor.
int ref_tc_method(int method, int64_t n, const int32_t* rp, const int32_t* col, uint64_t* count, double* ms) {
    try {
        Quiet q;
        std::vector<int> ones(rp[n], 1);
        lablas::Matrix<int> A;
        build(A, 0, n, rp, col, ones.data());
        LAGraph_Graph<int> graph(A);
        uint64_t ntri = 0;
        const double t0 = now_ms();
        lablas::algorithm::LAGr_TriangleCount(&ntri, &graph, (lablas::algorithm::LAGraph_TriangleCount_Method)method,
                                              lablas::algorithm::LAGraph_TriangleCount_NoSort,
                                              &lablas::GrB_DESC_IKJ_MASKED);
        if (ms) *ms = now_ms() - t0;
        *count = ntri;
        return 0;
    } catch (const char* e) {
        std::cerr << "reference error: " << e << std::endl;
        return 13;
    }
}

}  // extern "C"
