// Seeded synthetic graph generation (host side, OpenMP).
//
// Replaces the reference's time-seeded generators
// (src/helpers/graph_generation/graph_generation.hpp:93-191 RMAT,
//  :37-89 random_uniform, src/helpers/random_generator/common_generator/
//  common_generator.hpp:46-95) with a counter-based generator: every random
// draw is a pure function of (seed, stream, counter), so the same call gives
// the same graph on any machine and any thread count, and the CPU oracle and
// the GPU path are fed bit-identical CSR arrays.
//
// Random numbers: SplitMix64 output mixing (Steele, Lea, Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014) applied to
// key + (counter + 1) * golden-gamma.
//
// R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): each edge descends `scale`
// levels of the adjacency matrix; at each level it picks quadrant
// a=(0,0) b=(0,1) c=(1,0) d=(1,1) with 16-bit quantised probabilities.
// Like the reference generator, vertex labels are not permuted (hubs sit at
// low ids).  Self loops and duplicate edges are removed; undirected graphs
// add both directions before de-duplication.
//
// Output is CSR with int32 column ids, int32 row pointers (nnz < 2^31 is
// checked), columns sorted ascending within each row.

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "../../include/gbk_graphgen.h"

namespace {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ULL;

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
    return mix64(seed * kGamma + mix64(stream + 0x632BE59BD9B4E019ULL));
}

inline uint64_t draw(uint64_t key, uint64_t ctr) { return mix64(key + (ctr + 1) * kGamma); }

// Parallel LSD radix sort of 64-bit keys on the low `bits` bits, 8 bits per pass.
void radix_sort(std::vector<uint64_t>& a, int bits) {
    const size_t n = a.size();
    if (n < 2) return;
    std::vector<uint64_t> tmp(n);
    const int nthreads = omp_get_max_threads();
    std::vector<size_t> hist((size_t)nthreads * 256);
    uint64_t* src = a.data();
    uint64_t* dst = tmp.data();
    int passes = (bits + 7) / 8;
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nthreads)
        {
            const int t = omp_get_thread_num();
            const size_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
            size_t* h = &hist[(size_t)t * 256];
            for (size_t i = lo; i < hi; i++) h[(src[i] >> shift) & 0xFF]++;
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (int b = 0; b < 256; b++)
                    for (int tt = 0; tt < nthreads; tt++) {
                        size_t c = hist[(size_t)tt * 256 + b];
                        hist[(size_t)tt * 256 + b] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; i++) {
                uint64_t v = src[i];
                dst[h[(v >> shift) & 0xFF]++] = v;
            }
        }
        std::swap(src, dst);
    }
    if (src != a.data()) std::memcpy(a.data(), src, n * sizeof(uint64_t));
}

struct Graph {
    int64_t n = 0;
    int64_t nnz = 0;
    std::vector<int32_t> row_ptr;
    std::vector<int32_t> col;
};

// Sorted keys (src << vbits | dst) -> deduplicated CSR without self loops.
int keys_to_csr(std::vector<uint64_t>& keys, int vbits, int64_t n, Graph* g) {
    const uint64_t vmask = (vbits >= 64) ? ~0ULL : ((1ULL << vbits) - 1);
    radix_sort(keys, 2 * vbits);
    const size_t m = keys.size();
    const int nthreads = omp_get_max_threads();
    std::vector<size_t> cnt(nthreads + 1, 0);
    // keep[i]: first occurrence and not a self loop
    auto keep = [&](size_t i) {
        uint64_t k = keys[i];
        if ((k >> vbits) == (k & vmask)) return false;
        return i == 0 || keys[i - 1] != k;
    };
#pragma omp parallel num_threads(nthreads)
    {
        const int t = omp_get_thread_num();
        const size_t lo = m * t / nthreads, hi = m * (t + 1) / nthreads;
        size_t c = 0;
        for (size_t i = lo; i < hi; i++) c += keep(i);
        cnt[t + 1] = c;
    }
    for (int t = 0; t < nthreads; t++) cnt[t + 1] += cnt[t];
    const size_t nnz = cnt[nthreads];
    if (nnz >= (size_t)INT32_MAX) return GBK_GEN_TOO_LARGE;
    g->n = n;
    g->nnz = (int64_t)nnz;
    g->col.resize(nnz);
    std::vector<int32_t> row_of(nnz);
#pragma omp parallel num_threads(nthreads)
    {
        const int t = omp_get_thread_num();
        const size_t lo = m * t / nthreads, hi = m * (t + 1) / nthreads;
        size_t o = cnt[t];
        for (size_t i = lo; i < hi; i++)
            if (keep(i)) {
                g->col[o] = (int32_t)(keys[i] & vmask);
                row_of[o] = (int32_t)(keys[i] >> vbits);
                o++;
            }
    }
    g->row_ptr.assign(n + 1, 0);
    // row_ptr[r] = first index with row_of >= r (rows are sorted)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)nnz; i++) {
        int32_t r = row_of[i];
        int32_t prev = (i == 0) ? -1 : row_of[i - 1];
        for (int32_t q = prev + 1; q <= r; q++) g->row_ptr[q] = (int32_t)i;
    }
    int32_t last = nnz ? row_of[nnz - 1] : -1;
    for (int64_t q = last + 1; q <= n; q++) g->row_ptr[q] = (int32_t)nnz;
    return GBK_GEN_OK;
}

int emit(Graph& g, gbk_graph** out) {
    gbk_graph* h = (gbk_graph*)std::calloc(1, sizeof(gbk_graph));
    if (!h) return GBK_GEN_NO_MEMORY;
    h->n = g.n;
    h->nnz = g.nnz;
    h->row_ptr = (int32_t*)std::malloc(sizeof(int32_t) * (g.n + 1));
    h->col = (int32_t*)std::malloc(sizeof(int32_t) * (g.nnz ? g.nnz : 1));
    if (!h->row_ptr || !h->col) {
        std::free(h->row_ptr);
        std::free(h->col);
        std::free(h);
        return GBK_GEN_NO_MEMORY;
    }
    std::memcpy(h->row_ptr, g.row_ptr.data(), sizeof(int32_t) * (g.n + 1));
    if (g.nnz) std::memcpy(h->col, g.col.data(), sizeof(int32_t) * g.nnz);
    *out = h;
    return GBK_GEN_OK;
}

}  // namespace

extern "C" {

int gbk_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int undirected,
                 gbk_graph** out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 0) return GBK_GEN_BAD_ARG;
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12) return GBK_GEN_BAD_ARG;
    const int64_t n = 1LL << scale;
    const int64_t m = (int64_t)edge_factor * n;
    const uint32_t ta = (uint32_t)std::lround(a * 65536.0);
    const uint32_t tab = (uint32_t)std::lround((a + b) * 65536.0);
    const uint32_t tabc = (uint32_t)std::lround((a + b + c) * 65536.0);
    const uint64_t key = stream_key(seed, 1);
    const int words = (scale + 3) / 4;
    std::vector<uint64_t> keys((size_t)m * (undirected ? 2 : 1));
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) {
        uint64_t s = 0, d = 0, r = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 3) == 0) r = draw(key, (uint64_t)e * words + (l >> 2));
            uint32_t p = (uint32_t)(r & 0xFFFF);
            r >>= 16;
            uint64_t sb = (p >= tab) ? 1 : 0;
            uint64_t db = (p >= ta && p < tab) || (p >= tabc) ? 1 : 0;
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        if (undirected) {
            keys[2 * e] = (s << scale) | d;
            keys[2 * e + 1] = (d << scale) | s;
        } else {
            keys[e] = (s << scale) | d;
        }
    }
    Graph g;
    int rc = keys_to_csr(keys, scale, n, &g);
    if (rc) return rc;
    return emit(g, out);
}

int gbk_gen_uniform(int scale, int edge_factor, uint64_t seed, int undirected, gbk_graph** out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 0) return GBK_GEN_BAD_ARG;
    const int64_t n = 1LL << scale;
    const int64_t m = (int64_t)edge_factor * n;
    const uint64_t key = stream_key(seed, 2);
    std::vector<uint64_t> keys((size_t)m * (undirected ? 2 : 1));
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) {
        uint64_t r = draw(key, (uint64_t)e);
        uint64_t s = r >> (64 - scale);
        uint64_t d = (r >> (32 - scale)) & ((1ULL << scale) - 1);
        if (undirected) {
            keys[2 * e] = (s << scale) | d;
            keys[2 * e + 1] = (d << scale) | s;
        } else {
            keys[e] = (s << scale) | d;
        }
    }
    Graph g;
    int rc = keys_to_csr(keys, scale, n, &g);
    if (rc) return rc;
    return emit(g, out);
}

int gbk_gen_from_edges(int64_t n, int64_t m, const int64_t* src, const int64_t* dst, int undirected,
                       gbk_graph** out) {
    if (!out || n < 1 || m < 0 || (m > 0 && (!src || !dst))) return GBK_GEN_BAD_ARG;
    int vbits = 1;
    while ((1LL << vbits) < n) vbits++;
    if (vbits > 31) return GBK_GEN_TOO_LARGE;
    std::vector<uint64_t> keys((size_t)m * (undirected ? 2 : 1));
    for (int64_t e = 0; e < m; e++) {
        if (src[e] < 0 || src[e] >= n || dst[e] < 0 || dst[e] >= n) return GBK_GEN_BAD_ARG;
        uint64_t s = (uint64_t)src[e], d = (uint64_t)dst[e];
        if (undirected) {
            keys[2 * e] = (s << vbits) | d;
            keys[2 * e + 1] = (d << vbits) | s;
        } else {
            keys[e] = (s << vbits) | d;
        }
    }
    Graph g;
    int rc = keys_to_csr(keys, vbits, n, &g);
    if (rc) return rc;
    return emit(g, out);
}

void gbk_graph_free(gbk_graph* g) {
    if (!g) return;
    std::free(g->row_ptr);
    std::free(g->col);
    std::free(g);
}

// Edge value of (i, j) depends only on the unordered pair, so undirected
// graphs get symmetric values and the value does not depend on edge order.
static inline uint64_t pair_hash(uint64_t key, int64_t i, int64_t j) {
    uint64_t lo = (uint64_t)(i < j ? i : j), hi = (uint64_t)(i < j ? j : i);
    return draw(key, (lo << 32) | hi);
}

void gbk_gen_values_f32(int64_t n, const int32_t* row_ptr, const int32_t* col, uint64_t seed, float* out) {
    const uint64_t key = stream_key(seed, 3);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; i++)
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; e++)
            out[e] = (float)(pair_hash(key, i, col[e]) >> 40) * (1.0f / 16777216.0f);
}

void gbk_gen_weights_i32(int64_t n, const int32_t* row_ptr, const int32_t* col, uint64_t seed, int32_t lo,
                         int32_t hi, int32_t* out) {
    const uint64_t key = stream_key(seed, 4);
    const uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; i++)
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; e++)
            out[e] = lo + (int32_t)(((pair_hash(key, i, col[e]) >> 32) * span) >> 32);
}

void gbk_gen_vector_f32(int64_t n, uint64_t seed, float* out) {
    const uint64_t key = stream_key(seed, 5);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) out[i] = (float)(draw(key, (uint64_t)i) >> 40) * (1.0f / 16777216.0f);
}

int64_t gbk_gen_sources(int64_t n, const int32_t* row_ptr, int64_t count, uint64_t seed, int32_t* out) {
    const uint64_t key = stream_key(seed, 6);
    int64_t got = 0;
    for (uint64_t ctr = 0; got < count && ctr < (uint64_t)(64 * (count + n)); ctr++) {
        int64_t v = (int64_t)(((draw(key, ctr) >> 32) * (uint64_t)n) >> 32);
        if (row_ptr[v + 1] > row_ptr[v]) out[got++] = (int32_t)v;
    }
    return got;
}

// Matrix Market coordinate file of an edge list in the given order (1-based
// ids; a "%g" value column when vals != NULL), like the reference's
// EdgeListContainer::save_as_mtx (src/helpers/graph_generation/
// edges_container.hpp) except that the entries are not re-sorted.  Lines are
// formatted in parallel into per-thread buffers, then written in order.
int gbk_gen_write_mtx(const char* path, int64_t nrows, int64_t ncols, int64_t nnz, const int32_t* src,
                      const int32_t* dst, const float* vals) {
    FILE* fp = fopen(path, "wb");
    if (!fp) return GBK_GEN_BAD_ARG;
    fprintf(fp, "%%%%MatrixMarket matrix coordinate %s general\n%% written by gbk_gen_write_mtx\n%lld %lld %lld\n",
            vals ? "real" : "pattern", (long long)nrows, (long long)ncols, (long long)nnz);
    const int64_t block = 1 << 20;  // entries per formatting block
    const int64_t nblocks = (nnz + block - 1) / block;
    int rc = GBK_GEN_OK;
    for (int64_t b0 = 0; b0 < nblocks && rc == GBK_GEN_OK; b0 += 64) {
        const int64_t b1 = std::min<int64_t>(nblocks, b0 + 64);
        std::vector<std::string> out(b1 - b0);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t b = b0; b < b1; b++) {
            std::string& o = out[b - b0];
            o.reserve(block * 24);
            char line[96];
            for (int64_t e = b * block; e < std::min(nnz, (b + 1) * block); e++) {
                const int len = vals ? snprintf(line, sizeof(line), "%d %d %g\n", src[e] + 1, dst[e] + 1, (double)vals[e])
                                     : snprintf(line, sizeof(line), "%d %d\n", src[e] + 1, dst[e] + 1);
                o.append(line, (size_t)len);
            }
        }
        for (auto& o : out)
            if (fwrite(o.data(), 1, o.size(), fp) != o.size()) rc = GBK_GEN_BAD_ARG;
    }
    if (fclose(fp) != 0) rc = GBK_GEN_BAD_ARG;
    return rc;
}

// The reference's binary edge list (.mtxbin, read by binary_read_mtx_file,
// src/backend/matrix/read_file.hpp:377-400): int64 rows, cols, nnz, then nnz
// int64 (src, dst) pairs, 1-based.
int gbk_gen_write_mtxbin(const char* path, int64_t nrows, int64_t ncols, int64_t nnz, const int32_t* src,
                         const int32_t* dst) {
    FILE* fp = fopen(path, "wb");
    if (!fp) return GBK_GEN_BAD_ARG;
    int64_t h[3] = {nrows, ncols, nnz};
    int rc = fwrite(h, sizeof(h), 1, fp) == 1 ? GBK_GEN_OK : GBK_GEN_BAD_ARG;
    std::vector<int64_t> buf;
    const int64_t block = 1 << 22;
    for (int64_t e0 = 0; e0 < nnz && rc == GBK_GEN_OK; e0 += block) {
        const int64_t e1 = std::min(nnz, e0 + block);
        buf.resize(2 * (e1 - e0));
#pragma omp parallel for schedule(static)
        for (int64_t e = e0; e < e1; e++) {
            buf[2 * (e - e0)] = (int64_t)src[e] + 1;
            buf[2 * (e - e0) + 1] = (int64_t)dst[e] + 1;
        }
        if (fwrite(buf.data(), sizeof(int64_t), buf.size(), fp) != buf.size()) rc = GBK_GEN_BAD_ARG;
    }
    if (fclose(fp) != 0) rc = GBK_GEN_BAD_ARG;
    return rc;
}

}  // extern "C"
