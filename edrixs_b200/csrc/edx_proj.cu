// edx_proj.cu -- the final-state start vectors of the batched RIXS from stored projections:
// edx_proj_combine.
//
// The reference forms x_z per shift z (src/linsys.f90:3-128) and applies D_out^+ to it
// (src/rixs_driver.f90).  The batched solve keeps, for every Lanczos column c of H_n, the
// projected vectors D_out(p)^+ v_i (i < m) and the MINRES coefficients y of each shift in
// that column's basis, so D_out(p)^+ x_z = sum_i y_{z,i} D_out(p)^+ v_i: per (p, c) one
// complex product (shifts x m) times (m x rows).  This kernel writes it straight into the
// row-major block of final-state start vectors (rows x (p, c, shift) columns) that the
// final-state Lanczos reads.  FP64 on the CUDA cores (the fifth-generation tensor cores have
// no FP64 kind): 64 x 64 output tiles, 8 Lanczos vectors per shared-memory stage, every
// thread 4 rows x 4 shifts.  Each output is one sum over i in order, so results do not depend
// on the launch.
#include "edx_spmm.cuh"

namespace edx {

constexpr int PC_R = 64;    // rows per tile
constexpr int PC_W = 64;    // shifts per tile
constexpr int PC_I = 8;     // Lanczos vectors per stage
constexpr int PC_NT = 256;  // 16 x 16 threads

// out[r * ld_out + col0 + w] = sum_{i < m} y[w * ldy + i] * src[i * nrows + r]
// for r < nrows, w < nw (src: m rows of length nrows; y: nw rows of length >= m)
__global__ void __launch_bounds__(PC_NT, 2) k_proj_combine(const double2* __restrict__ src, int64_t nrows, int m,
                                                           const double2* __restrict__ y, int64_t ldy, int nw,
                                                           double2* __restrict__ out, int64_t ld_out,
                                                           int64_t col0) {
    __shared__ double2 sW[PC_I][PC_R];
    __shared__ double2 sY[PC_I][PC_W];
    const int tw = threadIdx.x % 16, tr = threadIdx.x / 16;  // shift group (consecutive lanes), row group
    const int64_t r0 = (int64_t)blockIdx.x * PC_R;
    const int w0 = blockIdx.y * PC_W;
    double2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = make_double2(0.0, 0.0);
    for (int i0 = 0; i0 < m; i0 += PC_I) {
        for (int e = threadIdx.x; e < PC_I * PC_R; e += PC_NT) {
            const int ii = e / PC_R, rr = e % PC_R;
            const int64_t r = r0 + rr;
            const int i = i0 + ii;
            sW[ii][rr] = (i < m && r < nrows) ? __ldg(src + (int64_t)i * nrows + r) : make_double2(0.0, 0.0);
        }
        for (int e = threadIdx.x; e < PC_I * PC_W; e += PC_NT) {
            const int ww = e / PC_I, ii = e % PC_I;
            const int w = w0 + ww, i = i0 + ii;
            sY[ii][ww] = (i < m && w < nw) ? __ldg(y + (int64_t)w * ldy + i) : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll
        for (int ii = 0; ii < PC_I; ++ii) {
            double2 wv[4], yv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) wv[a] = sW[ii][tr + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) yv[b] = sY[ii][tw + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma_c(yv[b], wv[a], acc[a][b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int64_t r = r0 + tr + 16 * a;
        if (r >= nrows) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int w = w0 + tw + 16 * b;
            if (w < nw) out[r * ld_out + col0 + w] = acc[a][b];
        }
    }
}

}  // namespace edx

using namespace edx;

extern "C" int edx_proj_combine(int np, const double* const* d_proj, int k, int maxn, int m, int64_t nrows,
                                const double* d_y, int64_t ldy, int nw, double* d_out, int64_t ld_out, void* stream) {
    EDX_REQUIRE(np >= 1 && d_proj != nullptr && k >= 1 && maxn >= 1 && m >= 1 && m <= maxn && nrows >= 1 &&
                    d_y != nullptr && ldy >= m && nw >= 1 && d_out != nullptr,
                "edx_proj_combine: bad arguments");
    EDX_REQUIRE(ld_out >= (int64_t)np * k * nw, "edx_proj_combine: ld_out %lld < np * k * nw = %lld",
                (long long)ld_out, (long long)np * k * nw);
    for (int p = 0; p < np; ++p) EDX_REQUIRE(d_proj[p] != nullptr, "edx_proj_combine: projection %d missing", p);
    cudaStream_t st = as_stream(stream);
    const int64_t rt = (nrows + PC_R - 1) / PC_R;
    EDX_REQUIRE(rt <= 0x7fffffff, "edx_proj_combine: too many rows");
    dim3 grid((unsigned)rt, (unsigned)((nw + PC_W - 1) / PC_W));
    for (int p = 0; p < np; ++p) {
        for (int c = 0; c < k; ++c) {
            const double2* src = reinterpret_cast<const double2*>(d_proj[p]) + (int64_t)c * maxn * nrows;
            const double2* yc = reinterpret_cast<const double2*>(d_y) + (int64_t)c * nw * ldy;
            k_proj_combine<<<grid, PC_NT, 0, st>>>(src, nrows, m, yc, ldy, nw, reinterpret_cast<double2*>(d_out),
                                                    ld_out, ((int64_t)p * k + c) * nw);
            EDX_CHECK_LAUNCH();
        }
    }
    return EDX_OK;
}
