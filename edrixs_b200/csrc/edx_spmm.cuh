// edx_spmm.cuh -- warp-per-row CSR x multi-vector core shared by the SpMM entry point and
// the fused Krylov / MINRES kernels.
#pragma once
#include "edx_common.cuh"

namespace edx {

// accumulate type: double unless both matrix and vectors are complex64
template <class VT, class XT>
struct Acc {
    using T = double2;
};
template <>
struct Acc<float2, float2> {
    using T = float2;
};

__device__ __forceinline__ double2 to_acc(double2 v, double2) { return v; }
__device__ __forceinline__ double2 to_acc(float2 v, double2) { return make_double2(v.x, v.y); }
__device__ __forceinline__ float2 to_acc(float2 v, float2) { return v; }

__device__ __forceinline__ double2 fma_c(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ float2 fma_c(float2 a, float2 b, float2 acc) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ double2 add_c(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 add_c(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 xor_sum(double2 v, int off) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
    return v;
}
__device__ __forceinline__ float2 xor_sum(float2 v, int off) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
    return v;
}
template <class T>
__device__ __forceinline__ T zero_c();
template <>
__device__ __forceinline__ double2 zero_c<double2>() { return make_double2(0.0, 0.0); }
template <>
__device__ __forceinline__ float2 zero_c<float2>() { return make_float2(0.f, 0.f); }

__device__ __forceinline__ double2 ldx(const double2* p) { return __ldg(p); }
__device__ __forceinline__ float2 ldx(const float2* p) { return __ldg(p); }

// Row r times column gc of X for a warp where lane = slot * KW + c (SLOTS = 32 / KW):
// the warp streams the row's nonzeros in chunks of 32 (one coalesced load per lane), then
// each slot takes every SLOTS-th entry of the chunk by shuffle.  Returns the full row sum in
// every lane of column c (slots reduced by xor-shuffles).
template <int KW, class VT, class XT>
__device__ __forceinline__ typename Acc<VT, XT>::T row_times_x(int64_t start, int64_t end,
                                                               const int32_t* __restrict__ col,
                                                               const VT* __restrict__ val,
                                                               const XT* __restrict__ X, int64_t ldx_,
                                                               int gc, bool colok) {
    using AT = typename Acc<VT, XT>::T;
    constexpr int SLOTS = 32 / KW;
    const int lane = threadIdx.x & 31;
    const int slot = lane / KW;
    AT acc = zero_c<AT>();
    if (KW == 1) {
        for (int64_t j = start + lane; j < end; j += 32) {
            int c = ld_stream(col + j);
            AT v = to_acc(ld_stream(val + j), AT());
            AT x = to_acc(ldx(X + (int64_t)c * ldx_ + gc), AT());
            acc = fma_c(v, x, acc);
        }
    } else {
        for (int64_t base = start; base < end; base += 32) {
            const int64_t j = base + lane;
            int cj = 0;
            VT vj;
            vj.x = 0;
            vj.y = 0;
            if (j < end) {
                cj = ld_stream(col + j);
                vj = ld_stream(val + j);
            }
            const int cnt = (end - base < 32) ? (int)(end - base) : 32;
#pragma unroll 4
            for (int t = 0; t < 32; t += SLOTS) {
                if (t >= cnt) break;
                const int src = t + slot;
                const int cc = __shfl_sync(0xffffffffu, cj, src);
                const VT vv = shfl2(vj, src);
                if (src < cnt && colok) {
                    AT x = to_acc(ldx(X + (int64_t)cc * ldx_ + gc), AT());
                    acc = fma_c(to_acc(vv, AT()), x, acc);
                }
            }
        }
    }
#pragma unroll
    for (int off = KW; off < 32; off <<= 1) acc = xor_sum(acc, off);
    return acc;
}

}  // namespace edx
