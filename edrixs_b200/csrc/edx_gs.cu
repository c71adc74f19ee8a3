// edx_gs.cu -- the two tall-skinny contractions of block Gram-Schmidt, for the thick-restart
// Lanczos eigensolver that replaces ARPACK (src/arpack.f90:2-112): C = V^H W and W -= V^T C,
// with V a set of m basis vectors (rows of length n) and W a block of k <= 8 vectors stored
// row-major (n x k).  Both are single passes over V at HBM speed; the dot keeps a
// deterministic summation order (per-block partials in fixed row chunks, then a fixed tree).
#include <algorithm>

#include "edx_common.cuh"

namespace edx {

namespace {

constexpr int GS_NT = 256;
constexpr int GS_NW = GS_NT / 32;
constexpr int GS_CHUNK = 512;  // rows of W staged per step (512 x 8 x 16 B = 64 KB at most)
constexpr int GS_KMAX = 8;

__device__ __forceinline__ double2 conj_mul(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// part[block][i][c] = sum over this block's row chunks of conj(V[i, r]) W[r, c]
template <int K>
__global__ void __launch_bounds__(GS_NT) k_gs_dot(int m, int64_t n, int64_t ldv, const double2* __restrict__ V,
                                                   const double2* __restrict__ W, double2* __restrict__ part) {
    extern __shared__ double2 gs_sm[];
    double2* wsm = gs_sm;                     // [GS_CHUNK][K]
    double2* acc_sm = gs_sm + GS_CHUNK * K;   // [m][K]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < m * K; t += GS_NT) acc_sm[t] = make_double2(0.0, 0.0);
    const int64_t nchunks = (n + GS_CHUNK - 1) / GS_CHUNK;
    for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        const int64_t r0 = ch * GS_CHUNK;
        const int nr = (int)((n - r0) < GS_CHUNK ? (n - r0) : GS_CHUNK);
        __syncthreads();
        for (int t = threadIdx.x; t < nr * K; t += GS_NT) wsm[t] = W[r0 * K + t];
        __syncthreads();
        for (int i = warp; i < m; i += GS_NW) {
            double2 acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = make_double2(0.0, 0.0);
            const double2* vi = V + (int64_t)i * ldv + r0;
            // four rows per lane per step: four loads in flight before the products
            for (int rb = 0; rb < nr; rb += 128) {
                double2 v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int rr = rb + q * 32 + lane;
                    v[q] = rr < nr ? __ldcs(vi + rr) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int rr = rb + q * 32 + lane;
                    if (rr < nr) {
#pragma unroll
                        for (int c = 0; c < K; ++c) {
                            const double2 p = conj_mul(v[q], wsm[rr * K + c]);
                            acc[c].x += p.x;
                            acc[c].y += p.y;
                        }
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < K; ++c)
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, off);
                    acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, off);
                }
            if (lane == 0) {
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    acc_sm[i * K + c].x += acc[c].x;
                    acc_sm[i * K + c].y += acc[c].y;
                }
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < m * K; t += GS_NT) part[(int64_t)blockIdx.x * m * K + t] = acc_sm[t];
}

// C[e] = sum over blocks of part[b][e]: a warp per entry, lanes over blocks, fixed tree
__global__ void k_gs_sum(int nb, int me, const double2* __restrict__ part, double2* __restrict__ C) {
    const int lane = threadIdx.x & 31;
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (e >= me) return;
    double2 s = make_double2(0.0, 0.0);
    for (int b = lane; b < nb; b += 32) {
        const double2 p = part[(int64_t)b * me + e];
        s.x += p.x;
        s.y += p.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, off);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, off);
    }
    if (lane == 0) C[e] = s;
}

// W[r, c] -= sum_i V[i, r] C[i, c]; a thread per row, C in shared memory
template <int K>
__global__ void __launch_bounds__(GS_NT) k_gs_update(int m, int64_t n, int64_t ldv, const double2* __restrict__ V,
                                                      double2* __restrict__ W, const double2* __restrict__ C) {
    extern __shared__ double2 c_sm[];  // [m][K]
    for (int t = threadIdx.x; t < m * K; t += GS_NT) c_sm[t] = C[t];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * GS_NT + threadIdx.x; r < n; r += (int64_t)gridDim.x * GS_NT) {
        double2 w[K];
#pragma unroll
        for (int c = 0; c < K; ++c) w[c] = W[r * K + c];
        for (int i = 0; i < m; ++i) {
            const double2 v = __ldcs(V + (int64_t)i * ldv + r);
#pragma unroll
            for (int c = 0; c < K; ++c) {
                const double2 q = c_sm[i * K + c];
                w[c].x -= v.x * q.x - v.y * q.y;
                w[c].y -= v.x * q.y + v.y * q.x;
            }
        }
#pragma unroll
        for (int c = 0; c < K; ++c) W[r * K + c] = w[c];
    }
}

// part[block][a][c] = sum over this block's rows of conj(W[r, a]) W[r, c] (the k x k Gram
// matrix of a row-major n x k block), then k_gs_sum; fixed row order per block
template <int K>
__global__ void __launch_bounds__(GS_NT) k_gs_gram(int64_t n, const double2* __restrict__ W,
                                                    double2* __restrict__ part) {
    __shared__ double2 red[GS_NW][K * K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2 acc[K * K];
#pragma unroll
    for (int e = 0; e < K * K; ++e) acc[e] = make_double2(0.0, 0.0);
    for (int64_t r = (int64_t)blockIdx.x * GS_NT + threadIdx.x; r < n; r += (int64_t)gridDim.x * GS_NT) {
        double2 w[K];
#pragma unroll
        for (int c = 0; c < K; ++c) w[c] = __ldcs(W + r * K + c);
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int c = 0; c < K; ++c) {
                const double2 p = conj_mul(w[a], w[c]);
                acc[a * K + c].x += p.x;
                acc[a * K + c].y += p.y;
            }
    }
#pragma unroll
    for (int e = 0; e < K * K; ++e)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            acc[e].x += __shfl_xor_sync(0xffffffffu, acc[e].x, off);
            acc[e].y += __shfl_xor_sync(0xffffffffu, acc[e].y, off);
        }
    if (lane == 0)
#pragma unroll
        for (int e = 0; e < K * K; ++e) red[warp][e] = acc[e];
    __syncthreads();
    for (int e = threadIdx.x; e < K * K; e += GS_NT) {
        double2 s = make_double2(0.0, 0.0);
        for (int q = 0; q < GS_NW; ++q) {
            s.x += red[q][e].x;
            s.y += red[q][e].y;
        }
        part[(int64_t)blockIdx.x * K * K + e] = s;
    }
}

// W = W M for a row-major n x k block and a k x k matrix M (row-major); a thread per row
template <int K>
__global__ void __launch_bounds__(GS_NT) k_gs_rmul(int64_t n, double2* __restrict__ W, const double2* __restrict__ M) {
    __shared__ double2 msm[K * K];
    for (int e = threadIdx.x; e < K * K; e += GS_NT) msm[e] = M[e];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * GS_NT + threadIdx.x; r < n; r += (int64_t)gridDim.x * GS_NT) {
        double2 w[K], o[K];
#pragma unroll
        for (int a = 0; a < K; ++a) {
            w[a] = W[r * K + a];
            o[a] = make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int a = 0; a < K; ++a)
#pragma unroll
            for (int c = 0; c < K; ++c) {
                const double2 q = msm[a * K + c];
                o[c].x += w[a].x * q.x - w[a].y * q.y;
                o[c].y += w[a].x * q.y + w[a].y * q.x;
            }
#pragma unroll
        for (int c = 0; c < K; ++c) W[r * K + c] = o[c];
    }
}

int gs_blocks() { return num_sms() * 4; }

template <template <int> class F, class... A>
int dispatch_k(int k, A... a) {
    switch (k) {
    case 1: return F<1>::run(a...);
    case 2: return F<2>::run(a...);
    case 3: return F<3>::run(a...);
    case 4: return F<4>::run(a...);
    case 5: return F<5>::run(a...);
    case 6: return F<6>::run(a...);
    case 7: return F<7>::run(a...);
    case 8: return F<8>::run(a...);
    }
    return fail(EDX_ERR_INVALID, "edx_gs: k must be 1..8");
}

template <int K>
struct DotRun {
    static int run(int m, int64_t n, int64_t ldv, const double2* V, const double2* W, double2* part, double2* C,
                   cudaStream_t st) {
        const size_t smem = sizeof(double2) * ((size_t)GS_CHUNK * K + (size_t)m * K);
        static bool attr[EDX_MAX_DEVICES] = {};
        int dev = 0;
        EDX_CUDA(cudaGetDevice(&dev));
        EDX_REQUIRE(dev >= 0 && dev < EDX_MAX_DEVICES, "edx_gs: device ordinal %d out of range", dev);
        if (!attr[dev]) {
            EDX_CUDA(cudaFuncSetAttribute(k_gs_dot<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr[dev] = true;
        }
        const int nb = gs_blocks();
        k_gs_dot<K><<<nb, GS_NT, smem, st>>>(m, n, ldv, V, W, part);
        EDX_CHECK_LAUNCH();
        const int me = m * K;
        k_gs_sum<<<(me * 32 + 255) / 256, 256, 0, st>>>(nb, me, part, C);
        EDX_CHECK_LAUNCH();
        return EDX_OK;
    }
};

template <int K>
struct UpdRun {
    static int run(int m, int64_t n, int64_t ldv, const double2* V, double2* W, const double2* C, cudaStream_t st) {
        const size_t smem = sizeof(double2) * (size_t)m * K;
        static bool attr[EDX_MAX_DEVICES] = {};
        int dev = 0;
        EDX_CUDA(cudaGetDevice(&dev));
        EDX_REQUIRE(dev >= 0 && dev < EDX_MAX_DEVICES, "edx_gs: device ordinal %d out of range", dev);
        if (!attr[dev]) {
            EDX_CUDA(cudaFuncSetAttribute(k_gs_update<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr[dev] = true;
        }
        const int64_t need = (n + GS_NT - 1) / GS_NT;
        const int nb = (int)std::min<int64_t>(need, (int64_t)num_sms() * 8);
        k_gs_update<K><<<nb, GS_NT, smem, st>>>(m, n, ldv, V, W, C);
        EDX_CHECK_LAUNCH();
        return EDX_OK;
    }
};

template <int K>
struct GramRun {
    static int run(int64_t n, const double2* W, double2* part, double2* G, cudaStream_t st) {
        const int nb = gs_blocks();
        k_gs_gram<K><<<nb, GS_NT, 0, st>>>(n, W, part);
        EDX_CHECK_LAUNCH();
        const int me = K * K;
        k_gs_sum<<<(me * 32 + 255) / 256, 256, 0, st>>>(nb, me, part, G);
        EDX_CHECK_LAUNCH();
        return EDX_OK;
    }
};

template <int K>
struct RmulRun {
    static int run(int64_t n, double2* W, const double2* M, cudaStream_t st) {
        const int64_t need = (n + GS_NT - 1) / GS_NT;
        const int nb = (int)std::min<int64_t>(need, (int64_t)num_sms() * 8);
        k_gs_rmul<K><<<nb, GS_NT, 0, st>>>(n, W, M);
        EDX_CHECK_LAUNCH();
        return EDX_OK;
    }
};

int check_gs(int m, int64_t n, int64_t ldv, int k, const void* V, const void* W, const void* C) {
    EDX_REQUIRE(V && W && C, "edx_gs: NULL pointer");
    EDX_REQUIRE(m >= 1 && n >= 1 && ldv >= n && k >= 1 && k <= GS_KMAX, "edx_gs: bad sizes");
    // shared memory: the C block (and the staged W chunk for the dot) must fit in 200 KB
    EDX_REQUIRE((size_t)(GS_CHUNK + m) * k * sizeof(double2) <= 200 * 1024,
                "edx_gs: m = %d basis vectors x k = %d is too large", m, k);
    return EDX_OK;
}

}  // namespace
}  // namespace edx

using namespace edx;

extern "C" int edx_gs_workspace(int m, int k, size_t* bytes) {
    EDX_REQUIRE(bytes && m >= 1 && k >= 1 && k <= GS_KMAX, "edx_gs_workspace: bad arguments");
    WorkspaceSize s;
    s.take<double2>((size_t)gs_blocks() * m * k);
    *bytes = s.bytes();
    return EDX_OK;
}

extern "C" int edx_gs_dot(const double* d_V, int m, int64_t n, int64_t ldv, const double* d_W, int k, double* d_C,
                          void* d_work, size_t work_bytes, void* stream) {
    int rc = check_gs(m, n, ldv, k, d_V, d_W, d_C);
    if (rc) return rc;
    Workspace w(d_work, work_bytes);
    double2* part = w.take<double2>((size_t)gs_blocks() * m * k);
    if (!part) return fail(EDX_ERR_WORKSPACE, "edx_gs_dot: workspace too small");
    return dispatch_k<DotRun>(k, m, n, ldv, reinterpret_cast<const double2*>(d_V),
                              reinterpret_cast<const double2*>(d_W), part, reinterpret_cast<double2*>(d_C),
                              as_stream(stream));
}

extern "C" int edx_gs_update(const double* d_V, int m, int64_t n, int64_t ldv, double* d_W, int k, const double* d_C,
                             void* stream) {
    int rc = check_gs(m, n, ldv, k, d_V, d_W, d_C);
    if (rc) return rc;
    return dispatch_k<UpdRun>(k, m, n, ldv, reinterpret_cast<const double2*>(d_V), reinterpret_cast<double2*>(d_W),
                              reinterpret_cast<const double2*>(d_C), as_stream(stream));
}

extern "C" int edx_gs_gram(const double* d_W, int64_t n, int k, double* d_G, void* d_work, size_t work_bytes,
                           void* stream) {
    EDX_REQUIRE(d_W && d_G && n >= 1 && k >= 1 && k <= GS_KMAX, "edx_gs_gram: bad arguments");
    Workspace w(d_work, work_bytes);
    double2* part = w.take<double2>((size_t)gs_blocks() * k * k);
    if (!part) return fail(EDX_ERR_WORKSPACE, "edx_gs_gram: workspace too small");
    return dispatch_k<GramRun>(k, n, reinterpret_cast<const double2*>(d_W), part, reinterpret_cast<double2*>(d_G),
                               as_stream(stream));
}

extern "C" int edx_gs_rmul(double* d_W, int64_t n, int k, const double* d_M, void* stream) {
    EDX_REQUIRE(d_W && d_M && n >= 1 && k >= 1 && k <= GS_KMAX, "edx_gs_rmul: bad arguments");
    return dispatch_k<RmulRun>(k, n, reinterpret_cast<double2*>(d_W), reinterpret_cast<const double2*>(d_M),
                               as_stream(stream));
}
