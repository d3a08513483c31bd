// Runs the reference's own algorithm files, unmodified, on the GPU library.
//
// The reference's algorithms/ headers are compiled against the drop-in header
// gb_kun_b200/dropin/src/gb_kun.h (the build recipe in this directory puts
// that src/ beside the reference's algorithms/ directory), so every
// lablas:: / GrB_* call they make runs as device kernels through libgbk.so.
// The calls below follow the reference's drivers: bfs.cpp:22-60, cc.cpp:83-117,
// pr.cpp:15-50, sssp.cpp:43-76, tc.cpp:33-70.
//
//   ref_algorithms <graph.bin> <out_dir> <source> <pr_iters>
//
// graph.bin: int64 n, int64 nnz, int32 row_ptr[n + 1], int32 col[nnz],
// int32 weight[nnz].  Each result goes to <out_dir>/<name>.bin as raw
// values; a line "name count" per result goes to stdout after "RESULTS".
#include "src/gb_kun.h"

#include "algorithms/bfs/bfs.hpp"
#include "algorithms/bfs/bfs_traditional.hpp"
#include "algorithms/cc/cc.hpp"
#include "algorithms/cc/cc_traditional.hpp"
#include "algorithms/pr/pr.hpp"
#include "algorithms/pr/pr_traditional.hpp"
#include "algorithms/sssp/sssp.hpp"
#include "algorithms/sssp/sssp_blast.hpp"
#include "algorithms/sssp/sssp_traditional.hpp"
#include "algorithms/tc/tc.hpp"

namespace {

struct Csr {
    int64_t n = 0, nnz = 0;
    std::vector<Index> row_ptr, col;
    std::vector<int> weight;
};

Csr read_graph(const char* path) {
    Csr g;
    FILE* f = std::fopen(path, "rb");
    if (!f) throw "cannot open the graph file";
    bool ok = std::fread(&g.n, 8, 1, f) == 1 && std::fread(&g.nnz, 8, 1, f) == 1;
    std::vector<int32_t> rp(g.n + 1), col(g.nnz);
    g.weight.resize(g.nnz);
    ok = ok && std::fread(rp.data(), 4, g.n + 1, f) == (size_t)(g.n + 1);
    ok = ok && std::fread(col.data(), 4, g.nnz, f) == (size_t)g.nnz;
    ok = ok && std::fread(g.weight.data(), 4, g.nnz, f) == (size_t)g.nnz;
    std::fclose(f);
    if (!ok) throw "truncated graph file";
    g.row_ptr.assign(rp.begin(), rp.end());
    g.col.assign(col.begin(), col.end());
    return g;
}

std::string g_out;
std::vector<std::pair<std::string, size_t>> g_written;

template <typename T>
void save(const std::string& name, const T* p, size_t count) {
    FILE* f = std::fopen((g_out + "/" + name + ".bin").c_str(), "wb");
    if (!f) throw "cannot write a result file";
    std::fwrite(p, sizeof(T), count, f);
    std::fclose(f);
    g_written.emplace_back(name, count);
}

template <typename T>
void save_vector(const std::string& name, lablas::Vector<T>& v) {
    // the reference's drivers read results through getDense()->get_vals()
    save(name, v.get_vector()->getDense()->get_vals(), (size_t)v.size());
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s graph.bin out_dir source pr_iters\n", argv[0]);
        return 2;
    }
    try {
        const Csr g = read_graph(argv[1]);
        g_out = argv[2];
        const Index source = std::atoll(argv[3]);
        const int pr_iters = std::atoi(argv[4]);

        std::vector<float> ones_f(g.nnz, 1.0f), w_f(g.weight.begin(), g.weight.end());
        std::vector<int> ones_i(g.nnz, 1);

        lablas::Descriptor desc;

        // BFS (bfs.cpp): float pattern matrix, bfs_blast, then the sequential checker
        {
            lablas::Matrix<float> matrix;
            matrix.set_preferred_matrix_format(CSR);
            matrix.build_from_csr_arrays(g.row_ptr.data(), g.col.data(), ones_f.data(), g.n, g.nnz);
            Index nrows;
            matrix.get_nrows(&nrows);
            lablas::Vector<float> levels(nrows);
            lablas::algorithm::bfs_blast(&levels, &matrix, source, &desc);
            save_vector("bfs_blast", levels);
            lablas::Vector<float> check_levels(nrows);
            lablas::algorithm::bfs_traditional(&check_levels, &matrix, source);
            save_vector("bfs_traditional", check_levels);
            std::cout << "bfs_blast equals bfs_traditional: " << (levels == check_levels) << std::endl;
        }
        // LAGraph-style BFS over a bool frontier and an int matrix (bfs.hpp:15-82)
        {
            lablas::Matrix<int> matrix;
            matrix.build_from_csr_arrays(g.row_ptr.data(), g.col.data(), ones_i.data(), g.n, g.nnz);
            LAGraph_Graph<int> graph(matrix);
            lablas::Vector<int>* level = nullptr;
            LG_BreadthFirstSearch_vanilla(&level, nullptr, &graph, source, false);
            save_vector("bfs_vanilla", *level);
            delete level;
        }
        // CC (cc.cpp): int matrix, the hooking mxv without SpMSpV as cc.cpp:2 sets
        {
            lablas::Matrix<int> matrix;
            matrix.build_from_csr_arrays(g.row_ptr.data(), g.col.data(), ones_i.data(), g.n, g.nnz);
            Index nrows;
            matrix.get_nrows(&nrows);
            lablas::Vector<int> components(nrows);
            {
                lablas::ScopedDisableSpMSpV no_spmspv;
                lablas::algorithm::cc(&components, &matrix, 0, &desc);
            }
            save_vector("cc", components);
            lablas::Vector<int> check_components(nrows);
            lablas::algorithm::cc_bfs_based_sequential(&check_components, &matrix);
            save_vector("cc_bfs_based_sequential", check_components);
        }
        // PageRank (pr.cpp): LAGraph_page_rank_sinks over LAGraph_Graph<float>
        {
            lablas::Matrix<float> matrix;
            matrix.build_from_csr_arrays(g.row_ptr.data(), g.col.data(), ones_f.data(), g.n, g.nnz);
            GrB_Index size;
            matrix.get_nrows(&size);
            LAGraph_Graph<float> graph(matrix);
            lablas::Vector<float> ranks(size);
            int iters_taken = 0;
            LAGraph_page_rank_sinks(&ranks, &graph, &iters_taken, pr_iters);
            save_vector("pr", ranks);
            lablas::Vector<float> check_ranks(size);
            lablas::algorithm::seq_page_rank(&check_ranks, &matrix, &iters_taken, pr_iters);
            save_vector("seq_page_rank", check_ranks);
        }
        // SSSP (sssp.cpp): float weights carrying integers, Bellman-Ford "blast",
        // the GraphBLAS Bellman-Ford and Dijkstra
        {
            lablas::Matrix<float> matrix;
            matrix.build_from_csr_arrays(g.row_ptr.data(), g.col.data(), w_f.data(), g.n, g.nnz);
            GrB_Index size;
            matrix.get_nrows(&size);
            LAGraph_Graph<float> graph(matrix);
            lablas::Vector<float> distances(size);
            lablas::algorithm::sssp_bellman_ford_blast(&distances, graph.A, source, &desc);
            save_vector("sssp_blast", distances);
            lablas::Vector<float> gbkun(size);
            lablas::algorithm::sssp_bellman_ford_gbkun(&gbkun, &matrix, source);
            save_vector("sssp_gbkun", gbkun);
            lablas::Vector<float> check_distances(size);
            lablas::algorithm::sssp_traditional_dijkstra(&check_distances, &matrix, source);
            save_vector("sssp_dijkstra", check_distances);
        }
        // Triangle counting (tc.cpp): LAGr_TriangleCount, default and Burkhardt
        // methods, both multiplication modes of the driver
        {
            lablas::Matrix<int> matrix;
            matrix.build_from_csr_arrays(g.row_ptr.data(), g.col.data(), ones_i.data(), g.n, g.nnz);
            LAGraph_Graph<int> graph(matrix);
            uint64_t counts[3] = {0, 0, 0};
            lablas::algorithm::LAGr_TriangleCount(&counts[0], &graph,
                                                  lablas::algorithm::LAGraph_TriangleCount_Default,
                                                  lablas::algorithm::LAGraph_TriangleCount_NoSort,
                                                  &lablas::GrB_DESC_IKJ_MASKED);
            lablas::algorithm::LAGr_TriangleCount(&counts[1], &graph,
                                                  lablas::algorithm::LAGraph_TriangleCount_Burkhardt,
                                                  lablas::algorithm::LAGraph_TriangleCount_NoSort,
                                                  &lablas::GrB_DESC_IJK_DOUBLE_SORT);
            // Cohen needs tricount_prep's lambda select: it must fail loudly here
            try {
                lablas::algorithm::LAGr_TriangleCount(&counts[2], &graph,
                                                      lablas::algorithm::LAGraph_TriangleCount_Cohen,
                                                      lablas::algorithm::LAGraph_TriangleCount_NoSort,
                                                      &lablas::GrB_DESC_IKJ_MASKED);
                counts[2] = 0;
            } catch (const char* e) {
                std::cout << "Cohen method: " << e << std::endl;
                counts[2] = 1;  // the lambda select was refused
            }
            save("tc", counts, 3);
        }
    } catch (const char* e) {
        std::cout << "error: " << e << std::endl;
        return 1;
    }
    std::cout << "RESULTS" << std::endl;
    for (auto& w : g_written) std::cout << w.first << " " << w.second << std::endl;
    return 0;
}
