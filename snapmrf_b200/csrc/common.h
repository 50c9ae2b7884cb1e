// Internal helpers shared by the snapMRF B200 library sources.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <string>

#include "snapmrf.h"

namespace snapmrf {

// Records `msg` as this thread's last error and returns `code`.
int set_error(int code, const char *fmt, ...);
void clear_error();
// Adds n to the process-wide kernel launch counter.
void note_launches(unsigned n);
// Counts one device scratch allocation (snapmrf_scratch_allocations).
void note_scratch_alloc();

}  // namespace snapmrf

#define SNAPMRF_FAIL(code, ...) return ::snapmrf::set_error((code), __VA_ARGS__)

#ifdef __CUDACC__
#include <cuda_runtime.h>

// Propagates a CUDA runtime failure as SNAPMRF_ERR_CUDA with its location.
#define SNAPMRF_CUDA(expr)                                                              \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess)                                                          \
            return ::snapmrf::set_error(_e == cudaErrorMemoryAllocation ? SNAPMRF_ERR_ALLOC \
                                                                        : SNAPMRF_ERR_CUDA, \
                                        "%s failed: %s (%s:%d)", #expr,                 \
                                        cudaGetErrorString(_e), __FILE__, __LINE__);    \
    } while (0)

#define SNAPMRF_LAUNCH_CHECK()            \
    do {                                  \
        ::snapmrf::note_launches(1);      \
        SNAPMRF_CUDA(cudaGetLastError()); \
    } while (0)

namespace snapmrf {

// Page-locked staging buffer of this thread on the current device for small
// uploads, so that cudaMemcpyAsync stays asynchronous.  stage_acquire waits
// for the previous upload from the buffer (stage_release records it).
void *stage_acquire(size_t bytes);
// Copies `bytes` from the staging buffer to device memory on `st` with a
// kernel that reads the page-locked host memory directly (no copy engine).
cudaError_t stage_upload(void *d_dst, const void *h_stage, size_t bytes, cudaStream_t st);
cudaError_t stage_release(cudaStream_t st);

// The library's stream-ordered memory pool on the current device.  Its
// release threshold is unlimited, so scratch freed by one call is reused by
// the next instead of being returned to the driver at every synchronisation
// (snapmrf_release_scratch trims it).
cudaError_t device_pool(cudaMemPool_t *pool);

// Stream-ordered scratch allocation that is released on scope exit.
struct DeviceScratch {
    void *ptr = nullptr;
    cudaStream_t stream = nullptr;
    DeviceScratch() = default;
    DeviceScratch(const DeviceScratch &) = delete;
    DeviceScratch &operator=(const DeviceScratch &) = delete;
    cudaError_t alloc(size_t bytes, cudaStream_t s) {
        stream = s;
        cudaMemPool_t pool;
        cudaError_t e = device_pool(&pool);
        if (e != cudaSuccess) return e;
        note_scratch_alloc();
        return cudaMallocFromPoolAsync(&ptr, bytes ? bytes : 16, pool, s);
    }
    ~DeviceScratch() {
        if (ptr) cudaFreeAsync(ptr, stream);
    }
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Complex helpers with the reference's float2 operator arithmetic
// (src/float2math.h:23-45): nvcc contracts them the same way.
__host__ __device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 c_scale(float2 a, float s) {
    return make_float2(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 c_add(float2 a, float2 b) {
    return make_float2(a.x + b.x, a.y + b.y);
}

}  // namespace snapmrf
#endif  // __CUDACC__
