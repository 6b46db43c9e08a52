// Shared helpers for the maos_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>
#include <string>
#include <vector>

#include "../../include/maos_b200.h"

namespace mb {

// Last error text for mb_last_error_message(); thread-local so concurrent
// reconstructors on different host threads do not overwrite each other.
void set_error(const char *fmt, ...);
const char *last_error();

// Counts kernels this library enqueued (direct launches plus graph nodes).
void count_launches(long n);

struct CudaError {
    int code;
};

#define MB_CUDA_TRY(call)                                                                  \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            mb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            throw mb::CudaError{MB_ECUDA};                                                 \
        }                                                                                  \
    } while (0)

#define MB_CHECK_LAUNCH()                                                                  \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess) {                                                           \
            mb::set_error("%s:%d kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            throw mb::CudaError{MB_ECUDA};                                                 \
        }                                                                                  \
        mb::count_launches(1);                                                             \
    } while (0)

struct InvalidArg {
    int code;
};
#define MB_REQUIRE(cond, ...)                                                              \
    do {                                                                                   \
        if (!(cond)) {                                                                     \
            mb::set_error(__VA_ARGS__);                                                    \
            throw mb::InvalidArg{MB_EINVAL};                                               \
        }                                                                                  \
    } while (0)

// Owning device buffer.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            set_error("cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
            throw CudaError{MB_ENOMEM};
        }
        n = count;
    }
    void upload(const std::vector<T> &h) {
        alloc(h.size());
        if (!h.empty()) MB_CUDA_TRY(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    void zero_async(cudaStream_t s) {
        if (p) MB_CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
};

}  // namespace mb
