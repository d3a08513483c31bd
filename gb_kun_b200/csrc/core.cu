// Library state: device selection, error text, launch accounting.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"
#include "internal.h"

namespace gbk {

static thread_local std::string g_error;
static std::atomic<int64_t> g_launches{0};
static int g_num_sms = 0;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    return GBK_CUDA_ERROR;
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

// add(3, 5) in the semiring's element type (src/backend/spmspv/spmspv.h:117).
int semiring_probe(int sr, int dtype) {
    (void)dtype;
    switch (sr) {
        case GBK_PLUS_TIMES:
        case GBK_PLUS_SECOND:
        case GBK_PLUS_ONE:
            return 8;
        case GBK_LOR_LAND:
        case GBK_STRUCTURAL_BOOL:
        case GBK_CUSTOM_LESS_PLUS:  // less(3, 5) == true
            return 1;
        default:  // min / first monoids
            return 3;
    }
}

}  // namespace gbk

extern "C" {

int gbk_init(int device) {
    int count = 0;
    GBK_CUDA(cudaGetDeviceCount(&count));
    GBK_REQUIRE(device >= 0 && device < count, GBK_INVALID_VALUE, "gbk_init: device %d of %d", device, count);
    GBK_CUDA(cudaSetDevice(device));
    cudaDeviceProp p;
    GBK_CUDA(cudaGetDeviceProperties(&p, device));
    GBK_REQUIRE(p.major == 10, GBK_UNSUPPORTED, "gbk_init: device %d is sm_%d%d, this library is built for sm_100a",
                device, p.major, p.minor);
    gbk::num_sms();
    // Temporaries come from the stream-ordered pool; keep freed blocks in this
    // process's pool instead of unmapping them at every synchronisation, which
    // would make the next allocation of a vector-sized buffer map pages again.
    cudaMemPool_t pool;
    GBK_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    GBK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    // Load the allocation-free entry point's code and scratch now, while
    // memory is free, instead of on its first call.
    return gbk::noalloc_setup(device);
}

int gbk_get_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return GBK_NULL_POINTER;
    std::strncpy(buf, gbk::g_error.c_str(), len - 1);
    buf[len - 1] = 0;
    return GBK_SUCCESS;
}

int64_t gbk_launch_count(void) { return gbk::g_launches.load(); }

}  // extern "C"
