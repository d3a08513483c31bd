/* CPU oracle (plain C restatement of the reference hot path).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg load this library, and only as the checker /
 * CPU baseline; the product library never links or calls it.
 *
 * Parity of this restatement is pinned against the reference's own CPU
 * code: tests/golden/ holds outputs of the reference library (built from its
 * sources by oracle/Makefile into oracle/_ref/) on seeded inputs, and
 * tests/test_oracle.py checks every function here against them. */
#include "oracle.h"

#include <float.h>
#include <stdio.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/gbk_types.h"

/* ---------------------------------------------------------------------- */
/* scalar semiring / operator semantics (src/cpp_graphblas/types.hpp:93-284) */

static double sr_identity(int sr, int dtype) {
    switch (sr) {
        case GBK_MIN_PLUS:
        case GBK_CUSTOM_LESS_PLUS:
        case GBK_MIN_SECOND:
        case GBK_MIN_NOTEQ:
            return dtype == ORC_F32 ? (double)FLT_MAX : (double)INT_MAX;
        default:
            return 0.0;
    }
}

/* Values are carried as double: exact for int32 and float operands.  Every
 * result is rounded back to the element type by `narrow`. */
static double narrow(double v, int dtype) {
    if (dtype == ORC_F32) return (double)(float)v;
    if (v >= (double)INT_MAX) return (double)INT_MAX;
    if (v <= (double)INT_MIN) return (double)INT_MIN;
    return (double)(int32_t)v;
}

/* Saturating integer add: INT_MAX (the min-plus identity) stays infinite. */
static double add_elem(double a, double b, int dtype) {
    if (dtype == ORC_F32) return (double)((float)a + (float)b);
    return narrow(a + b, dtype);
}

/* Integer multiply / subtract wrap modulo 2^32 as int32 arithmetic does in
 * the reference's C++ on two's-complement hardware. */
static double wrap_mul(double a, double b) {
    return (double)(int32_t)((uint32_t)(int32_t)a * (uint32_t)(int32_t)b);
}
static double wrap_sub(double a, double b) {
    return (double)(int32_t)((uint32_t)(int32_t)a - (uint32_t)(int32_t)b);
}

static double sr_add(int sr, double a, double b, int dtype) {
    switch (sr) {
        case GBK_PLUS_TIMES:
        case GBK_PLUS_SECOND:
        case GBK_PLUS_ONE:
            return add_elem(a, b, dtype);
        case GBK_LOR_LAND:
        case GBK_STRUCTURAL_BOOL:
            return (a != 0 || b != 0) ? 1.0 : 0.0;
        case GBK_FIRST_WINS:
            return a;
        case GBK_FIRST_MIN:
        case GBK_MIN_PLUS:
        case GBK_MIN_SECOND:
        case GBK_MIN_NOTEQ:
            return b < a ? b : a;
        case GBK_CUSTOM_LESS_PLUS:
            return a < b ? 1.0 : 0.0;
    }
    return 0.0;
}

static double sr_mul(int sr, double a, double x, int dtype) {
    switch (sr) {
        case GBK_PLUS_TIMES:
        case GBK_FIRST_WINS:
        case GBK_FIRST_MIN:
            return dtype == ORC_F32 ? (double)((float)a * (float)x) : wrap_mul(a, x);
        case GBK_LOR_LAND:
            return (a != 0 && x != 0) ? 1.0 : 0.0;
        case GBK_PLUS_SECOND:
        case GBK_MIN_SECOND:
            return x;
        case GBK_STRUCTURAL_BOOL:
        case GBK_PLUS_ONE:
            return 1.0;
        case GBK_MIN_PLUS:
        case GBK_CUSTOM_LESS_PLUS:
            return add_elem(a, x, dtype);
        case GBK_MIN_NOTEQ:
            return a != x ? 1.0 : 0.0;
    }
    return 0.0;
}

static double binop(int op, double a, double b, int dtype) {
    switch (op) {
        case GBK_OP_SECOND: return b;
        case GBK_OP_FIRST: return a;
        case GBK_OP_PLUS: return add_elem(a, b, dtype);
        case GBK_OP_MINUS: return dtype == ORC_F32 ? (double)((float)a - (float)b) : wrap_sub(a, b);
        case GBK_OP_TIMES: return dtype == ORC_F32 ? (double)((float)a * (float)b) : wrap_mul(a, b);
        case GBK_OP_DIV:
            if (dtype == ORC_F32) return (double)((float)a / (float)b);
            return b == 0 ? 0.0 : (double)((int32_t)a / (int32_t)b);
        case GBK_OP_MIN: return b < a ? b : a;
        case GBK_OP_MAX: return b > a ? b : a;
        case GBK_OP_LOR: return (a != 0 || b != 0) ? 1.0 : 0.0;
        case GBK_OP_LAND: return (a != 0 && b != 0) ? 1.0 : 0.0;
        case GBK_OP_NE: return a != b ? 1.0 : 0.0;
        case GBK_OP_LT: return a < b ? 1.0 : 0.0;
        case GBK_OP_ONE: return 1.0;
    }
    return b;
}

static double load(const void* p, int dtype, int64_t i) {
    return dtype == ORC_F32 ? (double)((const float*)p)[i] : (double)((const int32_t*)p)[i];
}

static void store(void* p, int dtype, int64_t i, double v) {
    if (dtype == ORC_F32)
        ((float*)p)[i] = (float)v;
    else
        ((int32_t*)p)[i] = (int32_t)v;
}

static int mask_true(const void* mask, int mask_dtype, int64_t i) {
    switch (mask_dtype) {
        case GBK_F32: return ((const float*)mask)[i] != 0.0f;
        case GBK_I32: return ((const int32_t*)mask)[i] != 0;
        case GBK_BOOL: return ((const uint8_t*)mask)[i] != 0;
        case GBK_I64: return ((const int64_t*)mask)[i] != 0;
        case GBK_F64: return ((const double*)mask)[i] != 0.0;
    }
    return 0;
}

/* ---------------------------------------------------------------------- */

void orc_spmv_f64(int64_t n, const int32_t* rp, const int32_t* col, const float* val, const float* x,
                  double* y) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        double s = 0.0;
        for (int64_t e = rp[i]; e < rp[i + 1]; e++) s += (double)val[e] * (double)x[col[e]];
        y[i] = s;
    }
}

int orc_mxv(int semiring, int accum, int dtype, int64_t n, const int32_t* rp, const int32_t* col,
            const void* val, const void* x, void* y, const void* mask, int mask_dtype, int mask_mode) {
    const double id = sr_identity(semiring, dtype);
    const int comp = (mask_mode == GBK_MASK_STR_COMP);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        if (mask) {
            int m = mask_true(mask, mask_dtype, i);
            if (!((!comp && m) || (comp && !m))) {
                store(y, dtype, i, 0.0); /* spmv_csr.h:324-327 */
                continue;
            }
        }
        double r = id;
        for (int64_t e = rp[i]; e < rp[i + 1]; e++)
            r = sr_add(semiring, r, sr_mul(semiring, load(val, dtype, e), load(x, dtype, col[e]), dtype), dtype);
        store(y, dtype, i, narrow(binop(accum, load(y, dtype, i), r, dtype), dtype));
    }
    return 0;
}

int orc_spmspv(int semiring, int accum, int dtype, int64_t n, const int32_t* rp, const int32_t* col,
               const void* val, int64_t nf, const int32_t* f_ids, const void* f_vals, void* y,
               const void* mask, int mask_dtype, int mask_mode) {
    const double id = sr_identity(semiring, dtype);
    /* kernel choice by probing add(3, 5) (spmspv.h:117-146) */
    double probe = sr_add(semiring, 3.0, 5.0, dtype);
    double* old = (double*)malloc(sizeof(double) * (n ? n : 1));
    if (!old) return 1;
    for (int64_t i = 0; i < n; i++) {
        old[i] = load(y, dtype, i);
        store(y, dtype, i, id);
    }
    for (int64_t k = 0; k < nf; k++) {
        int64_t i = f_ids[k];
        double xv = load(f_vals, dtype, k);
        for (int64_t e = rp[i]; e < rp[i + 1]; e++) {
            int64_t j = col[e];
            double a = load(val, dtype, e);
            double cur = load(y, dtype, j);
            double nv;
            if (probe == 8.0)
                nv = add_elem(cur, sr_mul(semiring, a, xv, dtype), dtype);
            else if (probe == 1.0)
                nv = 1.0;
            else
                nv = sr_add(semiring, cur, sr_mul(semiring, a, xv, dtype), dtype);
            store(y, dtype, j, nv);
        }
    }
    if (mask) { /* apply_mask, dense mask form (spmspv.h:17-70) */
        const int comp = (mask_mode == GBK_MASK_STR_COMP);
        for (int64_t i = 0; i < n; i++) {
            int m = mask_true(mask, mask_dtype, i);
            int active = comp ? !m : m;
            if (active)
                store(y, dtype, i, narrow(binop(accum, old[i], load(y, dtype, i), dtype), dtype));
            else
                store(y, dtype, i, 0.0);
        }
    }
    free(old);
    return 0;
}

/* ---------------------------------------------------------------------- */

void orc_bfs(int64_t n, const int32_t* rp, const int32_t* col, int32_t source, int32_t* levels) {
    int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    memset(levels, 0, sizeof(int32_t) * n);
    int64_t head = 0, tail = 0;
    levels[source] = 1;
    queue[tail++] = source;
    while (head < tail) {
        int32_t v = queue[head++];
        for (int64_t e = rp[v]; e < rp[v + 1]; e++) {
            int32_t u = col[e];
            if (!levels[u]) {
                levels[u] = levels[v] + 1;
                queue[tail++] = u;
            }
        }
    }
    free(queue);
}

static int32_t uf_find(int32_t* p, int32_t x) {
    while (p[x] != x) {
        p[x] = p[p[x]];
        x = p[x];
    }
    return x;
}

void orc_cc(int64_t n, const int32_t* rp, const int32_t* col, int32_t* labels) {
    int32_t* p = labels;
    for (int64_t i = 0; i < n; i++) p[i] = (int32_t)i;
    for (int64_t i = 0; i < n; i++)
        for (int64_t e = rp[i]; e < rp[i + 1]; e++) {
            int32_t a = uf_find(p, (int32_t)i), b = uf_find(p, col[e]);
            if (a != b) {
                if (a < b)
                    p[b] = a; /* the smaller id stays the root */
                else
                    p[a] = b;
            }
        }
    for (int64_t i = 0; i < n; i++) p[i] = uf_find(p, (int32_t)i);
}

/* binary heap keyed by distance */
typedef struct {
    int64_t d;
    int32_t v;
} hitem;

static void heap_push(hitem* h, int64_t* sz, hitem it) {
    int64_t i = (*sz)++;
    while (i > 0) {
        int64_t par = (i - 1) / 2;
        if (h[par].d <= it.d) break;
        h[i] = h[par];
        i = par;
    }
    h[i] = it;
}

static hitem heap_pop(hitem* h, int64_t* sz) {
    hitem top = h[0];
    hitem last = h[--(*sz)];
    int64_t i = 0;
    for (;;) {
        int64_t c = 2 * i + 1;
        if (c >= *sz) break;
        if (c + 1 < *sz && h[c + 1].d < h[c].d) c++;
        if (last.d <= h[c].d) break;
        h[i] = h[c];
        i = c;
    }
    h[i] = last;
    return top;
}

void orc_sssp(int64_t n, const int32_t* rp, const int32_t* col, const int32_t* w, int32_t source,
              int64_t* dist) {
    int64_t cap = rp[n] + 1;
    hitem* h = (hitem*)malloc(sizeof(hitem) * cap);
    int64_t sz = 0;
    for (int64_t i = 0; i < n; i++) dist[i] = -1;
    dist[source] = 0;
    hitem s = {0, source};
    heap_push(h, &sz, s);
    while (sz) {
        hitem it = heap_pop(h, &sz);
        if (it.d != dist[it.v]) continue;
        for (int64_t e = rp[it.v]; e < rp[it.v + 1]; e++) {
            int32_t u = col[e];
            int64_t nd = it.d + w[e];
            if (dist[u] < 0 || nd < dist[u]) {
                dist[u] = nd;
                hitem ni = {nd, u};
                heap_push(h, &sz, ni);
            }
        }
    }
    free(h);
}

/* Shared PageRank iteration: `seed` < 0 gives the global teleport of
 * pr.hpp:92-128, otherwise teleport and sink mass go to `seed`. */
static int pr_common(int64_t n, const int32_t* rp, const int32_t* col, int32_t seed, double damping,
                     double tol, int itermax, double* r, double* last_rdiff) {
    double* d = (double*)malloc(sizeof(double) * n);
    double* t = (double*)malloc(sizeof(double) * n);
    double* w = (double*)malloc(sizeof(double) * n);
    int64_t* cdeg = (int64_t*)calloc(n, sizeof(int64_t));
    /* d_out = G->coldegree (pr.hpp:37, cblas_wrappers/types.hpp:21-29) */
    for (int64_t e = 0; e < rp[n]; e++) cdeg[col[e]]++;
    for (int64_t i = 0; i < n; i++) {
        double dd = (double)cdeg[i] / damping;
        double dmin = 1.0 / damping;
        d[i] = dd > dmin ? dd : dmin; /* pr.hpp:84-90 */
    }
    const double scaled = (1.0 - damping) / (double)n;
    for (int64_t i = 0; i < n; i++) r[i] = (seed < 0) ? 1.0 / (double)n : (i == seed ? 1.0 : 0.0);
    /* The reference builds `sink` with a masked assign and lets it switch to
     * the sparse form when nsinks <= 0.3 n (vector.h:117-129).  Its masked
     * vector assign then reads u at the mask-list position instead of the
     * vertex id (generic_operations.h:28-34 with operations.h:63-65), so the
     * sink mass becomes the sum of the first nsinks ranks.  Restated as is. */
    int64_t nsinks = 0;
    for (int64_t i = 0; i < n; i++) nsinks += (cdeg[i] == 0);
    const int sparse_sink = seed < 0 && nsinks <= (int64_t)((double)n * 0.3);
    double rdiff = 1.0;
    int it;
    for (it = 0; it < itermax; it++) {
        double sink = 0.0;
        if (sparse_sink) {
            for (int64_t k = 0; k < nsinks; k++) sink += r[k];
        } else {
            for (int64_t i = 0; i < n; i++)
                if (cdeg[i] == 0) sink += r[i];
        }
        for (int64_t i = 0; i < n; i++) {
            t[i] = r[i];
            w[i] = t[i] / d[i];
        }
        if (seed < 0) {
            double teleport = scaled + damping / (double)n * sink;
            for (int64_t i = 0; i < n; i++) r[i] = teleport;
        } else {
            for (int64_t i = 0; i < n; i++) r[i] = 0.0;
            r[seed] = (1.0 - damping) + damping * sink;
        }
        for (int64_t i = 0; i < n; i++) {
            double s = 0.0;
            for (int64_t e = rp[i]; e < rp[i + 1]; e++) s += w[col[e]];
            r[i] += s;
        }
        rdiff = 0.0;
        for (int64_t i = 0; i < n; i++) rdiff += fabs(t[i] - r[i]);
        if (tol > 0 && rdiff < tol) {
            it++;
            break;
        }
    }
    if (last_rdiff) *last_rdiff = rdiff;
    free(d);
    free(t);
    free(w);
    free(cdeg);
    return it;
}

int orc_pagerank(int64_t n, const int32_t* rp, const int32_t* col, double damping, double tol, int itermax,
                 double* rank, double* last_rdiff) {
    return pr_common(n, rp, col, -1, damping, tol, itermax, rank, last_rdiff);
}

int orc_ppr(int64_t n, const int32_t* rp, const int32_t* col, int32_t seed, double damping, double tol,
            int itermax, double* rank) {
    return pr_common(n, rp, col, seed, damping, tol, itermax, rank, NULL);
}

uint64_t orc_tc(int64_t n, const int32_t* rp, const int32_t* col) {
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int64_t i = 0; i < n; i++) {
        for (int64_t e = rp[i]; e < rp[i + 1]; e++) {
            int32_t j = col[e];
            /* |N(i) ∩ N(j)| by merging two sorted rows */
            int64_t a = rp[i], ae = rp[i + 1], b = rp[j], be = rp[j + 1];
            while (a < ae && b < be) {
                if (col[a] < col[b])
                    a++;
                else if (col[a] > col[b])
                    b++;
                else {
                    total++;
                    a++;
                    b++;
                }
            }
        }
    }
    return total / 6;
}

void orc_transpose(int64_t n, const int32_t* rp, const int32_t* col, const float* val, int32_t* cp,
                   int32_t* row, float* tval) {
    memset(cp, 0, sizeof(int32_t) * (n + 1));
    for (int64_t e = 0; e < rp[n]; e++) cp[col[e] + 1]++;
    for (int64_t i = 0; i < n; i++) cp[i + 1] += cp[i];
    int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    for (int64_t i = 0; i < n; i++) pos[i] = cp[i];
    for (int64_t i = 0; i < n; i++)
        for (int64_t e = rp[i]; e < rp[i + 1]; e++) {
            int32_t q = pos[col[e]]++;
            row[q] = (int32_t)i;
            if (val && tval) tval[q] = val[e];
        }
    free(pos);
}

/* ------------------------------------------------------------------------ */
/* graph files (read_file.hpp:5-22, :27-47, :52-165, :377-400, :565-617)     */

static int orc_is_blank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

/* One data line: 0 = entry (ids 1-based in *a, *b), 1 = blank or comment,
 * 2 = malformed.  Accepts what sscanf("%lld %lld") accepts for non-negative
 * ids followed by a blank or the end of the line. */
static int orc_parse_line(const char* s, long long* a, long long* b) {
    const char* p = s;
    while (*p && orc_is_blank(*p)) p++;
    if (!*p || *p == '%') return 1;
    long long v[2] = {0, 0};
    for (int f = 0; f < 2; f++) {
        if (f) {
            if (!(*p == ' ' || *p == '\t')) return 2;
            while (*p == ' ' || *p == '\t') p++;
        }
        if (*p == '+') p++;
        int digits = 0;
        while (*p >= '0' && *p <= '9') {
            v[f] = v[f] * 10 + (*p - '0');
            if (++digits > 18) return 2;
            p++;
        }
        if (!digits) return 2;
    }
    if (*p && !orc_is_blank(*p)) return 2;
    *a = v[0];
    *b = v[1];
    return 0;
}

int orc_read_graph_file(const char* path, int kind, int64_t* nrows, int64_t* ncols, int64_t* nnz, int32_t* rp,
                        int32_t* col, int64_t* bad_line) {
    FILE* fp = fopen(path, kind == 0 ? "r" : "rb");
    if (!fp) return 1;
    long long r = 0, c = 0, z = 0;
    char line[8192];
    if (kind == 0) {
        int found = 0;
        while (fgets(line, sizeof(line), fp))
            if (line[0] != '%') {
                found = 1;
                break;
            }
        if (!found || sscanf(line, "%lld %lld %lld", &r, &c, &z) != 3 || r < 0 || c < 0 || z < 0) {
            fclose(fp);
            return 2;
        }
    } else {
        int64_t h[3];
        if (fread(h, sizeof(h), 1, fp) != 1 || h[0] < 0 || h[1] < 0 || h[2] < 0) {
            fclose(fp);
            return 2;
        }
        r = h[0];
        c = h[1];
        z = h[2];
    }
    *nrows = r;
    *ncols = c;
    *nnz = z;
    if (!rp) {
        fclose(fp);
        return 0;
    }
    int32_t* src = (int32_t*)malloc(sizeof(int32_t) * (size_t)(z > 0 ? z : 1));
    int32_t* dst = (int32_t*)malloc(sizeof(int32_t) * (size_t)(z > 0 ? z : 1));
    int rc = 0;
    int64_t got = 0, ln = 0;
    while (got < z) {
        long long a = 0, b = 0;
        if (kind == 0) {
            if (!fgets(line, sizeof(line), fp)) break;
            ln++;
            const int t = orc_parse_line(line, &a, &b);
            if (t == 1) continue;
            if (t == 2 || a < 1 || a > r || b < 1 || b > c) {
                rc = 3;
                if (bad_line) *bad_line = ln;
                break;
            }
        } else {
            int64_t pr[2];
            if (fread(pr, sizeof(pr), 1, fp) != 1) break;
            ln++;
            a = pr[0];
            b = pr[1];
            if (a < 1 || a > r || b < 1 || b > c) {
                rc = 3;
                if (bad_line) *bad_line = ln;
                break;
            }
        }
        src[got] = (int32_t)(a - 1);
        dst[got] = (int32_t)(b - 1);
        got++;
    }
    fclose(fp);
    if (rc == 0 && got < z) rc = 4;
    if (rc == 0) {
        /* counting sort by row: a row keeps the file order */
        for (int64_t i = 0; i <= r; i++) rp[i] = 0;
        for (int64_t e = 0; e < z; e++) rp[src[e] + 1]++;
        for (int64_t i = 0; i < r; i++) rp[i + 1] += rp[i];
        int32_t* fillp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(r > 0 ? r : 1));
        for (int64_t i = 0; i < r; i++) fillp[i] = rp[i];
        for (int64_t e = 0; e < z; e++) col[fillp[src[e]]++] = dst[e];
        free(fillp);
    }
    free(src);
    free(dst);
    return rc;
}
