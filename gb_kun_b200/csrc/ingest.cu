// Graph ingest: graph files parsed on the device into CSR, and a binary CSR
// cache.
//
// The reference reads a graph file on the host
// (src/backend/matrix/read_file.hpp): .mtx text line by line with fgets +
// sscanf (read_portion, :5-22) on one thread while a second pushes the pairs
// into per-row std::vectors (process_portion, :27-47; pipelined, :52-165),
// and .mtxbin with one fread and per-thread unordered_maps (:377-561); the
// CSR is then copied out of the vectors (vector_of_vectors_to_csr,
// src/helpers/lib_kernels/format_conversions.h:27-49).
//
// Here the host only moves bytes: the file is read in 8 MiB pieces by
// several pread threads into pinned buffers (two, so reading the next piece
// overlaps the device work on this one), each piece is cut at its last
// newline and copied to the device, and the device
//   * finds the line ends (a CUB select over the byte positions),
//   * parses each line with one thread (two 1-based ids; a value column,
//     blank lines and '%' lines are skipped),
//   * keeps the entry lines in file order (CUB select) and appends them to a
//     COO list, stopping at nnz entries as the reference reads nnz lines,
// then a stable radix sort by row gives the CSR with every row in file
// order (the order the reference's per-row push_back gives), the row
// pointers come from the row boundaries, and every value is 1 (EDGE_VAL).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "gbk_ingest.h"
#include "internal.h"

namespace gbk {
namespace {

constexpr int64_t kPieceBytesDefault = 8ll << 20;  // file bytes per read / parse step

// GBK_INGEST_PIECE_BYTES (at least 64) overrides the piece size, so small
// files can exercise the piece boundaries.
int64_t piece_bytes() {
    const char* e = getenv("GBK_INGEST_PIECE_BYTES");
    const long long v = e ? atoll(e) : 0;
    return v >= 64 ? (int64_t)v : kPieceBytesDefault;
}
constexpr int kReadThreadsDefault = 8;

// GBK_INGEST_READ_THREADS overrides the pread threads per piece (1 .. 64).
int read_threads() {
    const char* e = getenv("GBK_INGEST_READ_THREADS");
    const int v = e ? atoi(e) : 0;
    return v >= 1 && v <= 64 ? v : kReadThreadsDefault;
}
constexpr char kCsrMagic[8] = {'G', 'B', 'K', 'C', 'S', 'R', '0', '1'};
constexpr int64_t kCsrHeaderBytes = 64;

bool ends_with(const std::string& s, const char* e) {
    const size_t n = strlen(e);
    return s.size() >= n && s.compare(s.size() - n, n, e) == 0;
}

// The reference tells the kinds apart by the name's ending (read_file.hpp:570-586).
int kind_of(const char* path) {
    const std::string p(path);
    if (ends_with(p, ".gbkcsr")) return GBK_FILE_CSR;
    if (ends_with(p, "mtxbin")) return GBK_FILE_MTXBIN;
    if (ends_with(p, "mtx")) return GBK_FILE_MTX;
    return -1;
}

struct Fd {  // a file descriptor closed on scope exit
    int fd = -1;
    ~Fd() {
        if (fd >= 0) close(fd);
    }
};

// Read len bytes at offset off into dst with read_threads() pread threads;
// returns the bytes read (short only at the end of the file) or -1.
int64_t read_at(int fd, char* dst, int64_t off, int64_t len) {
    if (len <= 0) return 0;
    const int nt = len >= (4ll << 20) ? read_threads() : 1;
    std::vector<int64_t> got(nt, 0);
    auto work = [&](int t) {
        const int64_t a = len * t / nt, b = len * (t + 1) / nt;
        int64_t pos = a;
        while (pos < b) {
            const ssize_t r = pread(fd, dst + pos, (size_t)(b - pos), off + pos);
            if (r < 0) {
                got[t] = -1;
                return;
            }
            if (r == 0) break;
            pos += r;
        }
        got[t] = pos - a;
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    int64_t total = 0;
    for (int t = 0; t < nt; ++t) {
        if (got[t] < 0) return -1;
        total += got[t];
        // a short read inside the file (not at its end) leaves a hole
        if (got[t] < len * (t + 1) / nt - len * t / nt && t + 1 < nt && got[t + 1] > 0) return -1;
    }
    return total;
}

// ---------------------------------------------------------------------------
// device side

struct IsNewline {
    const char* t;
    __device__ bool operator()(const int32_t& i) const { return t[i] == '\n'; }
};

__device__ __forceinline__ bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// One thread per line: line k is [nl[k-1] + 1, nl[k]).  keep = 1 for an
// entry line with ids in range (src / dst 0-based); blank and '%' lines keep
// 0; a malformed line or an id out of range keeps 0 and lowers *bad to its
// index.
__global__ void k_parse_lines(const char* __restrict__ t, const int32_t* __restrict__ nl, const int32_t* nlines_p,
                              int64_t nrows, int64_t ncols, int32_t* __restrict__ src, int32_t* __restrict__ dst,
                              uint8_t* __restrict__ keep, int32_t* bad) {
    const int32_t nlines = *nlines_p;
    const int32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlines) return;
    int32_t i = k ? nl[k - 1] + 1 : 0;
    const int32_t end = nl[k];
    keep[k] = 0;
    while (i < end && is_blank(t[i])) ++i;
    if (i == end || t[i] == '%') return;
    unsigned long long id[2] = {0, 0};
    bool ok = true;
    for (int f = 0; f < 2 && ok; ++f) {
        if (f) {  // at least one blank between the ids
            if (i == end || !is_blank(t[i])) ok = false;
            while (i < end && is_blank(t[i])) ++i;
        }
        if (ok && i < end && t[i] == '+') ++i;
        int digits = 0;
        while (ok && i < end && t[i] >= '0' && t[i] <= '9') {
            id[f] = id[f] * 10 + (unsigned)(t[i] - '0');
            if (++digits > 18) ok = false;
            ++i;
        }
        if (digits == 0) ok = false;
    }
    // what follows the second id must start with a blank (a value column) or end the line
    if (ok && i < end && !is_blank(t[i])) ok = false;
    if (ok && (id[0] < 1 || id[0] > (unsigned long long)nrows || id[1] < 1 || id[1] > (unsigned long long)ncols))
        ok = false;
    if (!ok) {
        atomicMin(bad, k);
        return;
    }
    src[k] = (int32_t)(id[0] - 1);
    dst[k] = (int32_t)(id[1] - 1);
    keep[k] = 1;
}

// .mtxbin pairs (int64, 1-based) -> 0-based int32; *bad = the first pair out
// of range, numbered from the start of the file (first = this piece's start).
__global__ void k_bin_pairs(const int64_t* __restrict__ p, int64_t npairs, int64_t first, int64_t nrows,
                            int64_t ncols, int32_t* __restrict__ src, int32_t* __restrict__ dst, int64_t* bad) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npairs) return;
    const int64_t a = p[2 * k], b = p[2 * k + 1];
    if (a < 1 || a > nrows || b < 1 || b > ncols) {
        atomicMin((unsigned long long*)bad, (unsigned long long)(first + k));
        src[k] = 0;
        dst[k] = 0;
        return;
    }
    src[k] = (int32_t)(a - 1);
    dst[k] = (int32_t)(b - 1);
}

// Row pointers of rows sorted ascending: ptr[r] = first entry of row >= r.
__global__ void k_row_bounds(const int32_t* __restrict__ row, int64_t nnz, int64_t nrows, int32_t* __restrict__ ptr) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nnz) return;
    const int64_t lo = i == 0 ? 0 : (int64_t)row[i - 1] + 1;  // rows after the previous entry's ...
    const int64_t hi = i == nnz ? nrows : (int64_t)row[i];    // ... up to this entry's row start here
    for (int64_t r = lo; r <= hi; ++r) ptr[r] = (int32_t)i;
}

template <typename T>
__global__ void k_fill(T* __restrict__ v, int64_t n, T x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = x;
}

// A loaded CSR must be well formed before any kernel indexes with it:
// ptr[0] = 0, ptr non-decreasing, ptr[n] = nnz, columns in [0, ncols).
__global__ void k_check_csr(const int32_t* __restrict__ ptr, const int32_t* __restrict__ col, int64_t nrows,
                            int64_t ncols, int64_t nnz, int32_t* bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= nrows) {
        const int32_t p = ptr[i];
        if ((i == 0 && p != 0) || (i == nrows && p != nnz) || (i > 0 && p < ptr[i - 1]) || p < 0 || p > nnz)
            atomicExch(bad, 1);
    }
    if (i < nnz && (col[i] < 0 || col[i] >= ncols)) atomicExch(bad, 2);
}

unsigned nblocks(int64_t n) { return (unsigned)((n + 255) / 256); }

// ---------------------------------------------------------------------------
// headers

int mtx_header(const char* path, gbk_file_info* info) {
    FILE* fp = fopen(path, "r");
    GBK_REQUIRE(fp, GBK_INVALID_VALUE, "can not open graph file %s", path);
    char line[4096];
    int64_t lines = 0;
    bool found = false;
    while (fgets(line, sizeof(line), fp)) {  // '%' lines, then the size line (read_file.hpp:64-76)
        ++lines;
        if (line[0] != '%') {
            found = true;
            break;
        }
    }
    const long long off = found ? (long long)ftello(fp) : -1;
    fclose(fp);
    GBK_REQUIRE(found, GBK_INVALID_VALUE, "%s: unexpected end of graph file before the size line", path);
    long long r = -1, c = -1, z = -1;
    GBK_REQUIRE(sscanf(line, "%lld %lld %lld", &r, &c, &z) == 3 && r >= 0 && c >= 0 && z >= 0, GBK_INVALID_VALUE,
                "%s: bad size line \"%.80s\"", path, line);
    info->nrows = r;
    info->ncols = c;
    info->nnz = z;
    info->data_offset = off;
    return GBK_SUCCESS;
}

int bin_header(const char* path, gbk_file_info* info) {
    Fd f;
    f.fd = open(path, O_RDONLY);
    GBK_REQUIRE(f.fd >= 0, GBK_INVALID_VALUE, "can not open graph file %s", path);
    int64_t h[3];
    GBK_REQUIRE(pread(f.fd, h, sizeof(h), 0) == (ssize_t)sizeof(h), GBK_INVALID_VALUE,
                "%s: unexpected end of binary file in the header", path);
    GBK_REQUIRE(h[0] >= 0 && h[1] >= 0 && h[2] >= 0, GBK_INVALID_VALUE, "%s: negative sizes in the header", path);
    info->nrows = h[0];
    info->ncols = h[1];
    info->nnz = h[2];
    info->data_offset = sizeof(h);
    return GBK_SUCCESS;
}

int csr_header(const char* path, gbk_file_info* info) {
    Fd f;
    f.fd = open(path, O_RDONLY);
    GBK_REQUIRE(f.fd >= 0, GBK_INVALID_VALUE, "can not open CSR cache %s", path);
    char h[kCsrHeaderBytes];
    GBK_REQUIRE(pread(f.fd, h, sizeof(h), 0) == (ssize_t)sizeof(h), GBK_INVALID_VALUE,
                "%s: unexpected end of CSR cache in the header", path);
    GBK_REQUIRE(memcmp(h, kCsrMagic, 8) == 0, GBK_INVALID_VALUE, "%s: not a CSR cache (bad magic)", path);
    int64_t s[3];
    int32_t vt;
    memcpy(s, h + 8, sizeof(s));
    memcpy(&vt, h + 32, sizeof(vt));
    GBK_REQUIRE(s[0] >= 0 && s[1] >= 0 && s[2] >= 0 && (vt == GBK_F32 || vt == GBK_I32), GBK_INVALID_VALUE,
                "%s: bad CSR cache header", path);
    info->nrows = s[0];
    info->ncols = s[1];
    info->nnz = s[2];
    info->vtype = vt;
    info->data_offset = kCsrHeaderBytes;
    return GBK_SUCCESS;
}

int read_info(const char* path, gbk_file_info* info) {
    GBK_REQUIRE(path && info, GBK_NULL_POINTER, "gbk_file_info_read: NULL argument");
    memset(info, 0, sizeof(*info));
    info->vtype = -1;
    const int kind = kind_of(path);
    GBK_REQUIRE(kind >= 0, GBK_UNSUPPORTED, "%s: unsupported graph file (.mtx, .mtxbin or .gbkcsr)", path);
    info->kind = kind;
    struct stat st;
    GBK_REQUIRE(stat(path, &st) == 0, GBK_INVALID_VALUE, "can not open graph file %s", path);
    info->file_bytes = (int64_t)st.st_size;
    const int rc = kind == GBK_FILE_MTX ? mtx_header(path, info)
                   : kind == GBK_FILE_MTXBIN ? bin_header(path, info)
                                             : csr_header(path, info);
    if (rc) return rc;
    GBK_REQUIRE(info->nrows < INT32_MAX && info->ncols < INT32_MAX && info->nnz < INT32_MAX, GBK_INVALID_VALUE,
                "%s: sizes must fit int32 indices (rows %lld, cols %lld, nnz %lld)", path, (long long)info->nrows,
                (long long)info->ncols, (long long)info->nnz);
    return GBK_SUCCESS;
}

// ---------------------------------------------------------------------------
// COO (device, file order) -> matrix

// Sort the entries by row (stable: a row keeps the file order), derive the
// row pointers and make the matrix with every value 1.
int coo_to_matrix(gbk_matrix* out, int64_t nrows, int64_t ncols, int64_t nnz, int32_t* src, int32_t* dst,
                  gbk_dtype vtype, cudaStream_t s) {
    int32_t *rows = nullptr, *cols = nullptr, *ptr = nullptr;
    void* val = nullptr;
    void* tmp = nullptr;
    const int64_t m = std::max<int64_t>(nnz, 1);
    auto cleanup = [&]() {
        cudaFree(rows);
        cudaFree(cols);
        cudaFree(ptr);
        cudaFree(val);
        cudaFree(tmp);
    };
    int rc = GBK_SUCCESS;
    if (cudaMalloc(&rows, 4 * m) || cudaMalloc(&cols, 4 * m) || cudaMalloc(&ptr, 4 * (nrows + 1)) ||
        cudaMalloc(&val, 4 * m)) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "graph file: device allocation", __FILE__, __LINE__);
    }
    if (nnz > 0) {
        int bits = 1;
        while ((1ll << bits) < nrows) ++bits;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, src, rows, dst, cols, (int)nnz, 0, bits, s);
        if (cudaMalloc(&tmp, std::max<size_t>(tb, 16))) {
            cleanup();
            return cuda_fail(cudaGetLastError(), "graph file: sort scratch", __FILE__, __LINE__);
        }
        cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tb, src, rows, dst, cols, (int)nnz, 0, bits, s);
        if (e != cudaSuccess) {
            cleanup();
            return cuda_fail(e, "graph file: sort by row", __FILE__, __LINE__);
        }
        count_launch(1);
    }
    k_row_bounds<<<nblocks(nnz + 1), 256, 0, s>>>(rows, nnz, nrows, ptr);
    count_launch(1);
    if (nnz > 0) {
        if (vtype == GBK_F32)
            k_fill<float><<<nblocks(nnz), 256, 0, s>>>((float*)val, nnz, 1.0f);
        else
            k_fill<int32_t><<<nblocks(nnz), 256, 0, s>>>((int32_t*)val, nnz, 1);
        count_launch(1);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "graph file: CSR kernels", __FILE__, __LINE__);
    }
    rc = gbk_matrix_create_csr(out, nrows, ncols, nnz, ptr, cols, val, vtype, 1, s);
    cudaStreamSynchronize(s);
    cleanup();
    return rc;
}

// Scratch of the piece pipeline: two pinned host buffers and two device
// text buffers (so the next piece's read and copy overlap this piece's
// parse), per-line arrays sized for the worst case of one line per byte.
struct Pieces {
    char* host[2] = {nullptr, nullptr};
    char* text[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr};
    int32_t *nl = nullptr, *src = nullptr, *dst = nullptr, *ksrc = nullptr, *kdst = nullptr, *kline = nullptr;
    uint8_t* keep = nullptr;
    int32_t* cnt = nullptr;  // [0] lines, [1] kept, [2] first bad line
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    ~Pieces() {
        for (int b = 0; b < 2; ++b) {
            cudaFreeHost(host[b]);
            cudaFree(text[b]);
            if (copied[b]) cudaEventDestroy(copied[b]);
        }
        cudaFree(nl);
        cudaFree(src);
        cudaFree(dst);
        cudaFree(ksrc);
        cudaFree(kdst);
        cudaFree(kline);
        cudaFree(keep);
        cudaFree(cnt);
        cudaFree(tmp);
    }
};

int read_mtx(gbk_matrix* out, const char* path, const gbk_file_info& info, gbk_dtype vtype, cudaStream_t s) {
    const int64_t nnz = info.nnz;
    Fd f;
    f.fd = open(path, O_RDONLY);
    GBK_REQUIRE(f.fd >= 0, GBK_INVALID_VALUE, "can not open graph file %s", path);
    int32_t *coo_src = nullptr, *coo_dst = nullptr;
    struct CooFree {
        int32_t** a;
        int32_t** b;
        ~CooFree() {
            cudaFree(*a);
            cudaFree(*b);
        }
    } coo_free{&coo_src, &coo_dst};
    GBK_CUDA(cudaMalloc(&coo_src, 4 * std::max<int64_t>(nnz, 1)));
    GBK_CUDA(cudaMalloc(&coo_dst, 4 * std::max<int64_t>(nnz, 1)));
    Pieces P;
    const int64_t kPieceBytes = piece_bytes();
    const int64_t cap = kPieceBytes + 1;  // + a closing newline for a last line without one
    for (int b = 0; b < 2; ++b) {
        GBK_CUDA(cudaHostAlloc(&P.host[b], cap, cudaHostAllocDefault));
        GBK_CUDA(cudaMalloc(&P.text[b], cap));
        GBK_CUDA(cudaEventCreateWithFlags(&P.copied[b], cudaEventDisableTiming));
    }
    GBK_CUDA(cudaMalloc(&P.nl, 4 * cap));
    GBK_CUDA(cudaMalloc(&P.src, 4 * cap));
    GBK_CUDA(cudaMalloc(&P.dst, 4 * cap));
    GBK_CUDA(cudaMalloc(&P.ksrc, 4 * cap));
    GBK_CUDA(cudaMalloc(&P.kdst, 4 * cap));
    GBK_CUDA(cudaMalloc(&P.kline, 4 * cap));
    GBK_CUDA(cudaMalloc(&P.keep, cap));
    GBK_CUDA(cudaMalloc(&P.cnt, 4 * 4));
    {
        size_t a = 0, b = 0;
        thrust::counting_iterator<int32_t> it(0);
        cub::DeviceSelect::If(nullptr, a, it, P.nl, P.cnt, (int)cap, IsNewline{P.text[0]}, s);
        cub::DeviceSelect::Flagged(nullptr, b, P.src, P.keep, P.ksrc, P.cnt + 1, (int)cap, s);
        P.tmp_bytes = std::max(a, b);
        GBK_CUDA(cudaMalloc(&P.tmp, std::max<size_t>(P.tmp_bytes, 16)));
    }
    int64_t filled = 0;            // entries appended so far
    int64_t lines_before = 0;      // data lines of earlier pieces
    int64_t file_pos = info.data_offset;
    int64_t carry = 0;             // bytes of an unfinished line at the start of the next host buffer
    // read piece 0
    auto fill = [&](int b, int64_t& len, bool& eof) -> int {
        const int64_t want = kPieceBytes - carry;
        const int64_t got = read_at(f.fd, P.host[b] + carry, file_pos, want);
        GBK_REQUIRE(got >= 0, GBK_INVALID_VALUE, "%s: read error", path);
        file_pos += got;
        len = carry + got;
        eof = got < want;
        return GBK_SUCCESS;
    };
    int cur = 0;
    int64_t len = 0;
    bool eof = false;
    int rc = fill(cur, len, eof);
    if (rc) return rc;
    while (filled < nnz) {
        GBK_REQUIRE(len > 0 || !eof || filled >= nnz, GBK_INVALID_VALUE,
                    "%s: unexpected end of graph file after %lld of %lld entries", path, (long long)filled,
                    (long long)nnz);
        // cut the piece after its last newline; the rest starts the next piece
        int64_t use = len;
        if (!eof) {
            const void* lastnl = memrchr(P.host[cur], '\n', (size_t)len);
            GBK_REQUIRE(lastnl, GBK_INVALID_VALUE, "%s: a line longer than %lld bytes", path, (long long)kPieceBytes);
            use = (const char*)lastnl - P.host[cur] + 1;
        } else if (use > 0 && P.host[cur][use - 1] != '\n') {
            P.host[cur][use++] = '\n';
        }
        const int64_t rest = len - use;
        // device: copy, line ends, parse, keep the entry lines in order
        GBK_CUDA(cudaMemcpyAsync(P.text[cur], P.host[cur], use, cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaEventRecord(P.copied[cur], s));
        GBK_CUDA(cudaMemsetAsync(P.cnt, 0, 8, s));
        GBK_CUDA(cudaMemsetAsync(P.cnt + 2, 0x7f, 4, s));
        GBK_CUDA(cudaMemsetAsync(P.keep, 0, use, s));  // the selects below run over `use` flags
        size_t tb = P.tmp_bytes;
        thrust::counting_iterator<int32_t> it(0);
        GBK_CUDA(cub::DeviceSelect::If(P.tmp, tb, it, P.nl, P.cnt, (int)use, IsNewline{P.text[cur]}, s));
        count_launch(1);
        k_parse_lines<<<nblocks(use), 256, 0, s>>>(P.text[cur], P.nl, P.cnt, info.nrows, info.ncols, P.src, P.dst,
                                                   P.keep, P.cnt + 2);
        GBK_LAUNCHED();
        tb = P.tmp_bytes;
        GBK_CUDA(cub::DeviceSelect::Flagged(P.tmp, tb, P.src, P.keep, P.ksrc, P.cnt + 1, (int)use, s));
        tb = P.tmp_bytes;
        GBK_CUDA(cub::DeviceSelect::Flagged(P.tmp, tb, P.dst, P.keep, P.kdst, P.cnt + 3, (int)use, s));
        tb = P.tmp_bytes;
        GBK_CUDA(cub::DeviceSelect::Flagged(P.tmp, tb, it, P.keep, P.kline, P.cnt + 3, (int)use, s));
        count_launch(3);
        // meanwhile the host reads the next piece into the other buffer
        const int nxt = cur ^ 1;
        int64_t nlen = 0;
        bool neof = eof;
        if (!eof) {
            GBK_CUDA(cudaEventSynchronize(P.copied[nxt]));  // its previous copy has left the buffer
            memcpy(P.host[nxt], P.host[cur] + use, (size_t)rest);
            carry = rest;
            rc = fill(nxt, nlen, neof);
            if (rc) return rc;
        }
        int32_t cnt[4];
        GBK_CUDA(cudaMemcpyAsync(cnt, P.cnt, sizeof(cnt), cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaStreamSynchronize(s));
        const int64_t kept = cnt[1];
        const int64_t take = std::min<int64_t>(kept, nnz - filled);
        // a bad line counts if it comes before the line holding the nnz-th entry
        int32_t last_line = INT32_MAX;
        if (take > 0 && take == nnz - filled) {
            GBK_CUDA(cudaMemcpy(&last_line, P.kline + take - 1, 4, cudaMemcpyDeviceToHost));
        }
        GBK_REQUIRE(cnt[2] == 0x7f7f7f7f || cnt[2] > last_line, GBK_INVALID_VALUE,
                    "%s: bad entry at data line %lld (malformed, or an id outside 1..%lld / 1..%lld)", path,
                    (long long)(lines_before + cnt[2] + 1), (long long)info.nrows, (long long)info.ncols);
        if (take > 0) {
            GBK_CUDA(cudaMemcpyAsync(coo_src + filled, P.ksrc, 4 * take, cudaMemcpyDeviceToDevice, s));
            GBK_CUDA(cudaMemcpyAsync(coo_dst + filled, P.kdst, 4 * take, cudaMemcpyDeviceToDevice, s));
            filled += take;
        }
        lines_before += cnt[0];
        if (filled >= nnz) break;
        GBK_REQUIRE(!eof, GBK_INVALID_VALUE, "%s: unexpected end of graph file after %lld of %lld entries", path,
                    (long long)filled, (long long)nnz);
        cur = nxt;
        len = nlen;
        eof = neof;
    }
    GBK_CUDA(cudaStreamSynchronize(s));
    return coo_to_matrix(out, info.nrows, info.ncols, nnz, coo_src, coo_dst, vtype, s);
}

int read_mtxbin(gbk_matrix* out, const char* path, const gbk_file_info& info, gbk_dtype vtype, cudaStream_t s) {
    const int64_t nnz = info.nnz;
    GBK_REQUIRE(info.file_bytes >= info.data_offset + 16 * nnz, GBK_INVALID_VALUE,
                "%s: unexpected end of binary file (%lld entries need %lld bytes)", path, (long long)nnz,
                (long long)(info.data_offset + 16 * nnz));
    Fd f;
    f.fd = open(path, O_RDONLY);
    GBK_REQUIRE(f.fd >= 0, GBK_INVALID_VALUE, "can not open graph file %s", path);
    int32_t *coo_src = nullptr, *coo_dst = nullptr;
    int64_t* bad = nullptr;
    struct Free {
        int32_t** a;
        int32_t** b;
        int64_t** c;
        ~Free() {
            cudaFree(*a);
            cudaFree(*b);
            cudaFree(*c);
        }
    } fr{&coo_src, &coo_dst, &bad};
    GBK_CUDA(cudaMalloc(&coo_src, 4 * std::max<int64_t>(nnz, 1)));
    GBK_CUDA(cudaMalloc(&coo_dst, 4 * std::max<int64_t>(nnz, 1)));
    GBK_CUDA(cudaMalloc(&bad, 8));
    GBK_CUDA(cudaMemsetAsync(bad, 0x7f, 8, s));
    Pieces P;
    const int64_t kPieceBytes = std::max<int64_t>(16, piece_bytes() / 16 * 16);
    const int64_t pairs_per_piece = kPieceBytes / 16;
    for (int b = 0; b < 2; ++b) {
        GBK_CUDA(cudaHostAlloc(&P.host[b], kPieceBytes, cudaHostAllocDefault));
        GBK_CUDA(cudaMalloc(&P.text[b], kPieceBytes));
        GBK_CUDA(cudaEventCreateWithFlags(&P.copied[b], cudaEventDisableTiming));
    }
    // pieces go out back to back: a buffer is refilled once its copy is done,
    // and the id check is read once at the end
    int cur = 0;
    for (int64_t done = 0; done < nnz; done += pairs_per_piece, cur ^= 1) {
        const int64_t k = std::min<int64_t>(pairs_per_piece, nnz - done);
        GBK_CUDA(cudaEventSynchronize(P.copied[cur]));
        GBK_REQUIRE(read_at(f.fd, P.host[cur], info.data_offset + 16 * done, 16 * k) == 16 * k, GBK_INVALID_VALUE,
                    "%s: read error", path);
        GBK_CUDA(cudaMemcpyAsync(P.text[cur], P.host[cur], 16 * k, cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaEventRecord(P.copied[cur], s));
        k_bin_pairs<<<nblocks(k), 256, 0, s>>>((const int64_t*)P.text[cur], k, done, info.nrows, info.ncols,
                                                coo_src + done, coo_dst + done, bad);
        GBK_LAUNCHED();
    }
    int64_t first_bad = 0;
    GBK_CUDA(cudaMemcpyAsync(&first_bad, bad, 8, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    GBK_REQUIRE(first_bad == 0x7f7f7f7f7f7f7f7fll, GBK_INVALID_VALUE,
                "%s: entry %lld has an id outside 1..%lld / 1..%lld", path, (long long)(first_bad + 1),
                (long long)info.nrows, (long long)info.ncols);
    return coo_to_matrix(out, info.nrows, info.ncols, nnz, coo_src, coo_dst, vtype, s);
}

// Copy file bytes [off, off + bytes) to device memory dst through the two
// pinned piece buffers (the read of one piece overlaps the copy of the other).
int stream_to_device(int fd, const char* path, int64_t off, int64_t bytes, char* dst, cudaStream_t s) {
    const int64_t piece = std::max<int64_t>(16, piece_bytes());
    Pieces P;
    for (int b = 0; b < 2; ++b) {
        GBK_CUDA(cudaHostAlloc(&P.host[b], std::min(piece, std::max<int64_t>(bytes, 1)), cudaHostAllocDefault));
        GBK_CUDA(cudaEventCreateWithFlags(&P.copied[b], cudaEventDisableTiming));
    }
    int cur = 0;
    for (int64_t done = 0; done < bytes; done += piece, cur ^= 1) {
        const int64_t k = std::min(piece, bytes - done);
        GBK_CUDA(cudaEventSynchronize(P.copied[cur]));  // the copy that last used this buffer is done
        GBK_REQUIRE(read_at(fd, P.host[cur], off + done, k) == k, GBK_INVALID_VALUE, "%s: read error", path);
        GBK_CUDA(cudaMemcpyAsync(dst + done, P.host[cur], k, cudaMemcpyHostToDevice, s));
        GBK_CUDA(cudaEventRecord(P.copied[cur], s));
    }
    GBK_CUDA(cudaStreamSynchronize(s));
    return GBK_SUCCESS;
}

int load_csr(gbk_matrix* out, const char* path, const gbk_file_info& info, cudaStream_t s) {
    const int64_t n = info.nrows, nnz = info.nnz;
    const int64_t bytes = 4 * (n + 1) + 8 * nnz;
    GBK_REQUIRE(info.file_bytes >= kCsrHeaderBytes + bytes, GBK_INVALID_VALUE,
                "%s: unexpected end of CSR cache (%lld bytes, %lld needed)", path, (long long)info.file_bytes,
                (long long)(kCsrHeaderBytes + bytes));
    Fd f;
    f.fd = open(path, O_RDONLY);
    GBK_REQUIRE(f.fd >= 0, GBK_INVALID_VALUE, "can not open CSR cache %s", path);
    char* d = nullptr;  // row pointers, column ids and values back to back, as in the file
    int32_t* bad = nullptr;
    struct DevFree {
        char** a;
        int32_t** b;
        ~DevFree() {
            cudaFree(*a);
            cudaFree(*b);
        }
    } df{&d, &bad};
    GBK_CUDA(cudaMalloc(&d, std::max<int64_t>(bytes, 16)));
    GBK_CUDA(cudaMalloc(&bad, 4));
    int rc = stream_to_device(f.fd, path, kCsrHeaderBytes, bytes, d, s);
    if (rc) return rc;
    const int32_t* ptr = (const int32_t*)d;
    const int32_t* col = ptr + n + 1;
    const void* val = col + nnz;
    // a cache is input: check it before any kernel indexes with it
    int32_t hb = 0;
    GBK_CUDA(cudaMemsetAsync(bad, 0, 4, s));
    k_check_csr<<<nblocks(std::max(n + 1, nnz)), 256, 0, s>>>(ptr, col, n, info.ncols, nnz, bad);
    GBK_LAUNCHED();
    GBK_CUDA(cudaMemcpyAsync(&hb, bad, 4, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    GBK_REQUIRE(hb == 0, GBK_INVALID_VALUE, "%s: corrupt CSR cache (%s)", path,
                hb == 1 ? "row pointers" : "column ids");
    return gbk_matrix_create_csr(out, n, info.ncols, nnz, ptr, col, val, (gbk_dtype)info.vtype, 1, s);
}

}  // namespace
}  // namespace gbk

using namespace gbk;

extern "C" {

int gbk_file_info_read(const char* path, gbk_file_info* info) { return read_info(path, info); }

int gbk_matrix_create_from_file(gbk_matrix* out, const char* path, gbk_dtype vtype, void* stream) {
    GBK_REQUIRE(out && path, GBK_NULL_POINTER, "gbk_matrix_create_from_file: NULL argument");
    gbk_file_info info;
    int rc = read_info(path, &info);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (info.kind == GBK_FILE_CSR) return load_csr(out, path, info, s);
    GBK_REQUIRE(vtype == GBK_F32 || vtype == GBK_I32, GBK_UNSUPPORTED,
                "gbk_matrix_create_from_file: values must be GBK_F32 or GBK_I32");
    return info.kind == GBK_FILE_MTX ? read_mtx(out, path, info, vtype, s) : read_mtxbin(out, path, info, vtype, s);
}

int gbk_matrix_save_csr(gbk_matrix A, const char* path, void* stream) {
    GBK_REQUIRE(A && path, GBK_NULL_POINTER, "gbk_matrix_save_csr: NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    const CsrView& v = A->csr;
    const int64_t n = v.nrows, nnz = v.nnz;
    std::vector<char> h(kCsrHeaderBytes + 4 * (n + 1) + 8 * nnz, 0);
    memcpy(h.data(), kCsrMagic, 8);
    const int64_t sz[3] = {n, v.ncols, nnz};
    const int32_t vt = A->vtype;
    memcpy(h.data() + 8, sz, sizeof(sz));
    memcpy(h.data() + 32, &vt, sizeof(vt));
    char* body = h.data() + kCsrHeaderBytes;
    GBK_CUDA(cudaMemcpyAsync(body, v.ptr, 4 * (n + 1), cudaMemcpyDeviceToHost, s));
    if (nnz > 0) {
        GBK_CUDA(cudaMemcpyAsync(body + 4 * (n + 1), v.idx, 4 * nnz, cudaMemcpyDeviceToHost, s));
        GBK_CUDA(cudaMemcpyAsync(body + 4 * (n + 1) + 4 * nnz, v.val, 4 * nnz, cudaMemcpyDeviceToHost, s));
    }
    GBK_CUDA(cudaStreamSynchronize(s));
    FILE* fp = fopen(path, "wb");
    GBK_REQUIRE(fp, GBK_INVALID_VALUE, "can not create CSR cache %s", path);
    const size_t w = fwrite(h.data(), 1, h.size(), fp);
    const int c = fclose(fp);
    GBK_REQUIRE(w == h.size() && c == 0, GBK_INVALID_VALUE, "%s: write error", path);
    return GBK_SUCCESS;
}

int gbk_matrix_download_csr(gbk_matrix A, int32_t* row_ptr, int32_t* col, void* val, void* stream) {
    GBK_REQUIRE(A, GBK_NULL_POINTER, "gbk_matrix_download_csr: NULL matrix");
    cudaStream_t s = (cudaStream_t)stream;
    const CsrView& v = A->csr;
    if (row_ptr) GBK_CUDA(cudaMemcpyAsync(row_ptr, v.ptr, 4 * (v.nrows + 1), cudaMemcpyDeviceToHost, s));
    if (col && v.nnz > 0) GBK_CUDA(cudaMemcpyAsync(col, v.idx, 4 * v.nnz, cudaMemcpyDeviceToHost, s));
    if (val && v.nnz > 0) GBK_CUDA(cudaMemcpyAsync(val, v.val, dtype_size(A->vtype) * v.nnz, cudaMemcpyDeviceToHost, s));
    GBK_CUDA(cudaStreamSynchronize(s));
    return GBK_SUCCESS;
}

int gbk_matrix_load_csr(gbk_matrix* out, const char* path, void* stream) {
    GBK_REQUIRE(out && path, GBK_NULL_POINTER, "gbk_matrix_load_csr: NULL argument");
    gbk_file_info info;
    memset(&info, 0, sizeof(info));
    struct stat st;
    GBK_REQUIRE(stat(path, &st) == 0, GBK_INVALID_VALUE, "can not open CSR cache %s", path);
    info.file_bytes = (int64_t)st.st_size;
    int rc = csr_header(path, &info);
    if (rc) return rc;
    GBK_REQUIRE(info.nrows < INT32_MAX && info.ncols < INT32_MAX && info.nnz < INT32_MAX, GBK_INVALID_VALUE,
                "%s: sizes must fit int32 indices", path);
    return load_csr(out, path, info, (cudaStream_t)stream);
}

}  // extern "C"
