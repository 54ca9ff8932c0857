// Shared host/device utilities of the decon_b200 library: status handling,
// error strings, complex arithmetic and launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/decon_b200.h"

namespace dk {

// ---- host-side error state ---------------------------------------------
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define DK_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            /* a refused call leaves its error as the thread's last error: */             \
            /* clear it, or the next launch check would report it again */                \
            (void)cudaGetLastError();                                                     \
            return ::dk::fail(DECON_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                \
        }                                                                                 \
    } while (0)

// Count of kernels launched by the library (decon_launch_count), for the
// benchmark's launch accounting.
void count_launch();
// n kernels launched at once (a CUDA graph replay counts its kernel nodes)
void count_launches(int64_t n);

#define DK_LAUNCHED()                                                                     \
    do {                                                                                  \
        ::dk::count_launch();                                                             \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess)                                                            \
            return ::dk::fail(DECON_ERR_CUDA, "kernel launch failed: %s (%s:%d)",         \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                \
    } while (0)

#define DK_TRY(expr)                                                                      \
    do {                                                                                  \
        int s_ = (expr);                                                                  \
        if (s_ != DECON_OK) return s_;                                                    \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Division by a run-time divisor 1 <= d < 2^16 of dividends 0 <= q < 2^16 as
// one multiply: with m = floor(2^32 / d) + 1, floor(q / d) = (q m) >> 32.
// (q m / 2^32 exceeds q / d by less than q / 2^32 < 2^-16, while a
// non-integer q / d lies at least 1 / d > 2^-16 below the next integer.)
// Index loops of the FFT kernels divide a flat thread index by a row length
// this way instead of with the integer-division sequence.
struct FastDiv {
    uint64_t m;
};
inline FastDiv make_fastdiv(int64_t d) { return FastDiv{(1ull << 32) / (uint64_t)d + 1}; }
__device__ __forceinline__ int fdiv(int q, FastDiv f) {
    return (int)(((uint64_t)(uint32_t)q * f.m) >> 32);
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return cdiv(a, b) * b; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Copy / fill device memory and return only once the bytes are in place,
// visible to work on every stream.  For set-up data that several streams may
// read (twiddle tables, fresh solver state): a plain cudaMemcpy from pageable
// memory or a cudaMemset runs on the legacy default stream, which does not
// order against non-blocking streams, and may still be in flight when another
// stream's kernel reads the buffer.  Uses a private non-blocking stream per
// device and synchronises only that stream.
int upload_blocking(void* dst, const void* src, size_t bytes);
int memset_blocking(void* dst, int value, size_t bytes);

// ---- complex helpers -------------------------------------------------------
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
    return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
    return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) {
    return make_float2(a.x * s, a.y * s);
}

// ---- FP64 block reduction ---------------------------------------------------
// Sum of one double per thread over the block; result valid in thread 0.
// blockDim.x must be a multiple of 32 and <= 1024.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < (unsigned)nw) ? red[threadIdx.x] : 0.0;
    if (warp == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace dk
