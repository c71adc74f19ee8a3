// edx_common.cuh -- shared device/host helpers for libedx (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/edx.h"

namespace edx {

// ------------------------------------------------------------------------------------
// error plumbing: every entry point returns a status and leaves a message behind
// ------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define EDX_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::edx::fail(EDX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,              \
                               cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

#define EDX_CHECK_LAUNCH()                                                                \
    do {                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess)                                                            \
            return ::edx::fail(EDX_ERR_CUDA, "kernel launch failed: %s (%s:%d)",          \
                               cudaGetErrorString(e_), __FILE__, __LINE__);               \
    } while (0)

#define EDX_REQUIRE(cond, ...)                                                            \
    do {                                                                                  \
        if (!(cond)) return ::edx::fail(EDX_ERR_INVALID, __VA_ARGS__);                    \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int num_sms();  // SM count of the current device (cached per device)

// bump allocator over a caller-provided workspace; every slice is 256-byte aligned
struct Workspace {
    char* base;
    size_t size;
    size_t used;
    Workspace(void* p, size_t n) : base(static_cast<char*>(p)), size(n), used(0) {}
    template <class T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        size_t bytes = count * sizeof(T);
        if (base == nullptr || off + bytes > size) return nullptr;
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};
// size accounting twin of Workspace::take
struct WorkspaceSize {
    size_t used = 0;
    template <class T>
    void take(size_t count) {
        used = ((used + 255) & ~size_t(255)) + count * sizeof(T);
    }
    size_t bytes() const { return used + 256; }
};

// ------------------------------------------------------------------------------------
// complex arithmetic (double2 / float2 = interleaved re, im)
// Division uses Smith's algorithm (R. L. Smith, CACM 5(8):435, 1962); the square root
// uses the half-angle identities for the principal branch.
// ------------------------------------------------------------------------------------
__host__ __device__ inline double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ inline double2 cadd(double2 a, double2 b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 csub(double2 a, double2 b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ inline double2 cmul(double2 a, double2 b) {
    return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ inline double2 cconjmul(double2 a, double2 b) {
    return cmk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ inline double2 cscale(double2 a, double s) { return cmk(a.x * s, a.y * s); }
__host__ __device__ inline double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ inline double cabs_(double2 a) { return hypot(a.x, a.y); }
__host__ __device__ inline double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double t = b.y / b.x, d = b.x + b.y * t;
        return cmk((a.x + a.y * t) / d, (a.y - a.x * t) / d);
    } else {
        double t = b.x / b.y, d = b.x * t + b.y;
        return cmk((a.x * t + a.y) / d, (a.y * t - a.x) / d);
    }
}
__host__ __device__ inline double2 csqrt_(double2 a) {
    double m = cabs_(a);
    if (m == 0.0) return cmk(0.0, 0.0);
    if (a.x >= 0.0) {
        double r = sqrt(0.5 * (m + a.x));
        return cmk(r, a.y / (2.0 * r));
    }
    double i = copysign(sqrt(0.5 * (m - a.x)), a.y);
    return cmk(a.y / (2.0 * i), i);
}

__host__ __device__ inline float2 cmkf(float r, float i) { return make_float2(r, i); }

// ------------------------------------------------------------------------------------
// warp helpers
// ------------------------------------------------------------------------------------
__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ inline double2 shfl2(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ inline float2 shfl2(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

__device__ inline unsigned lane_id() { return threadIdx.x & 31u; }

// streaming load for read-once matrix data: no L1 allocation, L2 evict-first policy
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double2 ld_stream(const double2* p) {
    double2 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                 : "=d"(v.x), "=d"(v.y)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}
__device__ __forceinline__ float2 ld_stream(const float2* p) {
    float2 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(v.x), "=f"(v.y)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}
// TMA bulk prefetch of bytes [begin, end) of `base` into L2.  The untiled bulk form needs a
// 16-byte aligned address and a size that is a multiple of 16: the range is widened to 16-byte
// boundaries and clamped to the last full 16-byte block below `limit` (the array's byte size),
// so it never reaches past the array.  A prefetch is a hint; nothing waits on it.
__device__ __forceinline__ void prefetch_l2(const void* base, int64_t begin, int64_t end, int64_t limit) {
    int64_t a0 = begin & ~int64_t(15);
    int64_t a1 = (end + 15) & ~int64_t(15);
    const int64_t lim = limit & ~int64_t(15);
    if (a1 > lim) a1 = lim;
    if (a1 <= a0) return;
    int64_t size = a1 - a0;
    if (size > (int64_t)1 << 20) size = (int64_t)1 << 20;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(static_cast<const char*>(base) + a0),
                 "r"((unsigned)size)
                 : "memory");
}

__device__ __forceinline__ int ld_stream(const int* p) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
                 : "=r"(v)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}

}  // namespace edx
