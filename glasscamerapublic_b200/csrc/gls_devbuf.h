// gls_devbuf.h — error-propagation macros and a growable device buffer,
// shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include "gls_host.h"

namespace gls {

#define GLS_CUDA(...)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (__VA_ARGS__);                                                                     \
        if (e_ != cudaSuccess)                                                                          \
            return set_error(e_ == cudaErrorMemoryAllocation ? GLS_ERR_OOM : GLS_ERR_CUDA, "%s: %s (%s:%d)", \
                             #__VA_ARGS__, cudaGetErrorString(e_), __FILE__, __LINE__);                        \
    } while (0)

#define GLS_TRY(...)                     \
    do {                                 \
        gls_status s_ = (__VA_ARGS__);   \
        if (s_ != GLS_OK) return s_;     \
    } while (0)

// Bytes of device memory the library holds (all of it is DevBuf), summed
// over devices, and the largest value since the last reset
// (gls_device_memory).
void devbuf_account(long long delta);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    gls_status ensure(size_t b) {
        if (b <= bytes) return GLS_OK;
        if (p) {
            cudaFree(p);
            devbuf_account(-static_cast<long long>(bytes));
        }
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            return set_error(GLS_ERR_OOM, "cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(e));
        }
        bytes = b;
        devbuf_account(static_cast<long long>(b));
        return GLS_OK;
    }
    // ensure(), and a newly allocated buffer is zeroed on stream s (a
    // buffer that its users leave zeroed after each use)
    gls_status ensure_zeroed(size_t b, cudaStream_t s) {
        if (b <= bytes) return GLS_OK;
        const gls_status st = ensure(b);
        if (st != GLS_OK) return st;
        const cudaError_t e = cudaMemsetAsync(p, 0, b, s);
        if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
        return GLS_OK;
    }
    void release() {
        if (p) {
            cudaFree(p);
            devbuf_account(-static_cast<long long>(bytes));
        }
        p = nullptr;
        bytes = 0;
    }
};

}  // namespace gls
