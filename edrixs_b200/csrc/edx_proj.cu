// edx_proj.cu -- the final-state start vectors of the batched RIXS from stored projections:
// edx_proj_combine.
//
// The reference forms x_z per shift z (src/linsys.f90:3-128) and applies D_out^+ to it
// (src/rixs_driver.f90).  The batched solve keeps, for every Lanczos column c of H_n, the
// projected vectors D_out(p)^+ v_i (i < m) and the MINRES coefficients y of each shift in
// that column's basis, so D_out(p)^+ x_z = sum_i y_{z,i} D_out(p)^+ v_i: per (p, c) one
// complex product (shifts x m) times (m x rows).  This kernel writes it straight into the
// row-major block of final-state start vectors (rows x (p, c, shift) columns) that the
// final-state Lanczos reads.  FP64 through the warp-level FP64 MMA (the fifth-generation
// tensor cores' tcgen05 instructions have no FP64 kind): 64 x 64 output tiles, 16 Lanczos
// vectors per shared-memory stage, every warp 32 rows x 16 shifts.  The summation order is
// fixed by the tiling, so results do not depend on the launch.
#include "edx_spmm.cuh"

namespace edx {

constexpr int PC_R = 64;    // rows per block tile
constexpr int PC_W = 64;    // shifts per block tile
constexpr int PC_I = 16;    // Lanczos vectors per shared-memory stage (4 MMA k-steps)
constexpr int PC_NT = 256;  // 8 warps: 2 (rows) x 4 (shifts), each 32 rows x 16 shifts

// D = A B + C for one 8 x 8 x 4 FP64 tile (warp-level MMA; lane l holds A[l/4][l%4],
// B[l%4][l/4] and C, D[l/4][2(l%4) + {0, 1}])
__device__ __forceinline__ void mma_f64(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// out[r * ld_out + col0 + w] = sum_{i < m} y[w * ldy + i] * src[i * nrows + r]
// for r < nrows, w < nw (src: m rows of length nrows; y: nw rows of length >= m).  As a
// matrix product C = A B with A[r][i] = src[i][r] and B[i][w] = y[w][i], complex, through
// four real FP64 MMAs per tile and k-step into separate real and imaginary accumulators.
__global__ void __launch_bounds__(PC_NT, 2) k_proj_combine(const double2* __restrict__ src, int64_t nrows, int m,
                                                           const double2* __restrict__ y, int64_t ldy, int nw,
                                                           double2* __restrict__ out, int64_t ld_out,
                                                           int64_t col0) {
    __shared__ double2 sW[PC_I][PC_R];
    __shared__ double2 sY[PC_I][PC_W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = warp >> 2, wc = warp & 3;          // warp tile: rows wr*32.., shifts wc*16..
    const int g = lane >> 2, q = lane & 3;            // MMA fragment coordinates
    const int64_t r0 = (int64_t)blockIdx.x * PC_R;
    const int w0 = blockIdx.y * PC_W;
    double cr[4][2][2], ci[4][2][2];                  // [row tile][shift tile][element]
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u) cr[t][u][0] = cr[t][u][1] = ci[t][u][0] = ci[t][u][1] = 0.0;
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
        for (int ks = 0; ks < PC_I / 4; ++ks) {
            double2 a[4], b[2];
#pragma unroll
            for (int t = 0; t < 4; ++t) a[t] = sW[ks * 4 + q][wr * 32 + t * 8 + g];
#pragma unroll
            for (int u = 0; u < 2; ++u) b[u] = sY[ks * 4 + q][wc * 16 + u * 8 + g];
#pragma unroll
            for (int t = 0; t < 4; ++t)
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    mma_f64(cr[t][u][0], cr[t][u][1], a[t].x, b[u].x);
                    mma_f64(cr[t][u][0], cr[t][u][1], -a[t].y, b[u].y);
                    mma_f64(ci[t][u][0], ci[t][u][1], a[t].x, b[u].y);
                    mma_f64(ci[t][u][0], ci[t][u][1], a[t].y, b[u].x);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int64_t r = r0 + wr * 32 + t * 8 + g;
        if (r >= nrows) continue;
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int w = w0 + wc * 16 + u * 8 + 2 * q + e;
                if (w < nw) out[r * ld_out + col0 + w] = make_double2(cr[t][u][e], ci[t][u][e]);
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
