// Device plumbing shared by the lablas:: headers: stream selection, status
// translation and typed device buffers.  Host code only: it calls the CUDA
// runtime C API and the gbk C ABI, never device code directly.
#pragma once

#include <cuda_runtime_api.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gbk.h"
#include "types.hpp"

namespace lablas {

// All lablas calls of a host thread are ordered on one CUDA stream
// (NULL = the legacy default stream).
inline cudaStream_t& current_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}
inline void set_stream(void* s) { current_stream() = (cudaStream_t)s; }
inline void* stream() { return (void*)current_stream(); }

inline std::string last_error() {
    char buf[1024];
    gbk_get_last_error(buf, sizeof(buf));
    return buf;
}

// gbk status -> LA_Info (identical numbering up to GrB_PANIC)
inline LA_Info to_info(int rc) {
    if (rc >= 0 && rc <= GrB_PANIC) return (LA_Info)rc;
    return GrB_PANIC;
}

// Errors where the reference throws `const char*` (constructors, conversions).
inline void throw_if(int rc, const char* where) {
    if (rc != 0) {
        static thread_local std::string msg;
        msg = std::string(where) + ": " + last_error();
        throw msg.c_str();
    }
}

inline void cuda_check(cudaError_t e, const char* where) {
    if (e != cudaSuccess) {
        static thread_local std::string msg;
        msg = std::string(where) + ": " + cudaGetErrorString(e);
        throw msg.c_str();
    }
}

template <typename T>
struct DeviceBuffer {
    T* p = nullptr;
    size_t n = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t count) { alloc(count); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }
    // stream-ordered: no device-wide synchronisation per temporary
    void alloc(size_t count) {
        static const int ready = [] {  // once per process: gbk_init sets up the pool on the current device
            int d = 0;
            cudaGetDevice(&d);
            return gbk_init(d);
        }();
        (void)ready;
        release();
        n = count;
        cuda_check(cudaMallocAsync((void**)&p, sizeof(T) * (count ? count : 1), current_stream()), "cudaMallocAsync");
    }
    void release() {
        if (p) cudaFreeAsync(p, current_stream());
        p = nullptr;
        n = 0;
    }
    void swap(DeviceBuffer& o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    void upload(const T* host, size_t count) {
        cuda_check(cudaMemcpyAsync(p, host, sizeof(T) * count, cudaMemcpyHostToDevice, current_stream()), "upload");
    }
    void download(T* host, size_t count) const {
        cuda_check(cudaMemcpyAsync(host, p, sizeof(T) * count, cudaMemcpyDeviceToHost, current_stream()),
                   "download");
        cuda_check(cudaStreamSynchronize(current_stream()), "download sync");
    }
    void copy_from(const DeviceBuffer& o, size_t count) {
        cuda_check(cudaMemcpyAsync(p, o.p, sizeof(T) * count, cudaMemcpyDeviceToDevice, current_stream()), "copy");
    }
};

// Vectors switch to the sparse form at this density (la_backend.h:11).
constexpr double SPARSE_VECTOR_THRESHOLD = 0.3;

}  // namespace lablas
