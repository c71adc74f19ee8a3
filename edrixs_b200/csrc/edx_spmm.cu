// edx_spmm.cu -- complex CSR SpMV / SpMM (kernels K7, K8).
//
// Y = alpha*(A X) + sigma*X + beta*Y over k right-hand sides.  matvec_csr
// (src/spmv.f90:73-103) is the k = 1, alpha = 1, beta = 1, sigma = 0 case (y += A x).  One
// warp per row; lanes are split into SLOTS = 32/KW slots x KW columns so that a row's
// nonzeros stream through the warp in coalesced 32-entry chunks (column indices and values
// each loaded once, with L1 no-allocate / L2 evict-first hints since the matrix is read
// once per product) while the gathered X rows stay L2-resident.  Column tiles of width KW
// run as grid.y so that wide blocks (k = 768) keep one X tile hot in L2 at a time.
#include <algorithm>

#include "edx_spmm.cuh"

namespace edx {

template <int KW, class VT, class XT, bool ROWSLOT, int HALF = 0>
__global__ void __launch_bounds__(256) k_spmm(int64_t nrows, const int64_t* __restrict__ row_ptr,
                                              const int32_t* __restrict__ col, const VT* __restrict__ val,
                                              int k, const XT* __restrict__ X, int64_t ldx_, XT* __restrict__ Y,
                                              int64_t ldy, int64_t ycs, double2 alpha, double2 sigma,
                                              double2 beta, int has_sigma, int has_beta) {
    using AT = typename Acc<VT, XT>::T;
    constexpr int SLOTS = Slots<KW>::N;
    const int lane = threadIdx.x & 31;
    const int c = lane % KW;
    const int slot = lane / KW;
    const int gc = blockIdx.y * KW + c;
    const bool colok = gc < k;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    auto store = [&](int64_t r, AT acc) {
        double yr = alpha.x * (double)acc.x - alpha.y * (double)acc.y;
        double yi = alpha.x * (double)acc.y + alpha.y * (double)acc.x;
        if (has_sigma) {
            XT xv = X[r * ldx_ + gc];
            yr += sigma.x * (double)xv.x - sigma.y * (double)xv.y;
            yi += sigma.x * (double)xv.y + sigma.y * (double)xv.x;
        }
        XT* yp = Y + r * ldy + (int64_t)gc * ycs;
        if (has_beta) {
            XT yv = *yp;
            yr += beta.x * (double)yv.x - beta.y * (double)yv.y;
            yi += beta.x * (double)yv.y + beta.y * (double)yv.x;
        }
        XT out;
        out.x = yr;
        out.y = yi;
        *yp = out;
    };
    if constexpr (KW == 1 && !ROWSLOT && HALF > 0) {  // one column, rows of <= ~100 entries: two per warp
        spmv_rows_half<HALF, VT, XT>(warp0, nw, nrows, row_ptr, col, val, X, ldx_, gc, [&](int64_t r, AT acc) {
            if ((lane & 15) == 0) store(r, acc);
        });
        return;
    } else if constexpr (KW == 1 && !ROWSLOT) {  // one column, long rows: the next row loads during this one
        spmv_rows<VT, XT>(warp0, nrows, nw, row_ptr, col, val, X, ldx_, gc, [&](int64_t r, AT acc) {
            if (lane == 0) store(r, acc);
        });
        return;
    } else {
        const int64_t rstep = ROWSLOT ? nw * SLOTS : nw;
        for (int64_t rb = ROWSLOT ? warp0 * SLOTS : warp0; rb < nrows; rb += rstep) {
            const int64_t r = ROWSLOT ? rb + slot : rb;
            AT acc;
            bool mine;
            if (ROWSLOT) {
                mine = slot < SLOTS && r < nrows;
                const int64_t s = mine ? __ldg(row_ptr + r) : 0, e = mine ? __ldg(row_ptr + r + 1) : 0;
                row_times_x_slot<KW, VT, XT>(s, e, col, val, X, ldx_, gc, colok, acc);
            } else {
                mine = lane < KW;
                const int64_t s = __ldg(row_ptr + r), e = __ldg(row_ptr + r + 1);
                AT accv[1];
                row_times_x_tiles<KW, 1, VT, XT>(s, e, col, val, X, ldx_, blockIdx.y * KW, k, accv);
                acc = accv[0];
            }
            if (mine && colok) store(r, acc);
        }
    }
}

// rows of at most this many entries on average run one row per slot
constexpr int64_t SHORT_ROW = 16;
// one-column products on rows of at most this many entries on average run two rows per warp
constexpr int64_t HALF_WARP_ROW = 100;
constexpr int64_t HALF_NC5_ROW = 75;  // up to this many: five entries per lane prefetched, else six

// resident blocks per SM of a kernel (cached per device): a grid-stride launch then runs as
// one wave with no tail of late blocks
// (one cache per kernel: the kernel is a template argument, so that instantiations with the
// same signature do not share an entry)
template <auto KERN>
static int resident_blocks(int threads) {
    static int cache[EDX_MAX_DEVICES] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= EDX_MAX_DEVICES) return 4;
    if (cache[dev] == 0) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, KERN, threads, 0) != cudaSuccess || nb < 1) nb = 4;
        cache[dev] = nb;
    }
    return cache[dev];
}

template <int NC, class VT, class XT>
static int launch_spmv_half(const edx_csr* A, const void* x, int64_t ldx_, void* y, int64_t ldy, int64_t ycs,
                            double2 al, double2 sg, double2 be, cudaStream_t st) {
    const int threads = 256;
    const int res = resident_blocks<k_spmm<1, VT, XT, false, NC>>(threads);
    const int64_t need = ((A->nrows + 1) / 2 * 32 + threads - 1) / threads;
    const int64_t bx = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)num_sms() * res));
    const int hs = (sg.x != 0.0 || sg.y != 0.0) ? 1 : 0;
    const int hb = (be.x != 0.0 || be.y != 0.0) ? 1 : 0;
    k_spmm<1, VT, XT, false, NC><<<dim3((unsigned)bx, 1), threads, 0, st>>>(
        A->nrows, A->row_ptr, A->col, reinterpret_cast<const VT*>(A->val), 1, reinterpret_cast<const XT*>(x), ldx_,
        reinterpret_cast<XT*>(y), ldy, ycs, al, sg, be, hs, hb);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <int KW, class VT, class XT>
static int launch_spmm_t(const edx_csr* A, int k, const void* x, int64_t ldx_, void* y, int64_t ldy,
                         int64_t ycs, double2 al, double2 sg, double2 be, cudaStream_t st) {
    const int threads = 256;
    // a row per slot for short rows at any width below 32, and for 6-16 columns at any row
    // length: no reduction across slots per row (H_n, 6 columns: 1.13 ms against 1.65 ms with
    // a warp per row; at 3 columns the two were level)
    const bool rowslot = KW < 32 && (A->nnz <= SHORT_ROW * A->nrows || (KW >= 6 && KW <= 16));
    if (KW == 1 && !rowslot && A->nnz <= HALF_WARP_ROW * A->nrows) {  // two rows per warp
        if (A->nnz <= HALF_NC5_ROW * A->nrows) return launch_spmv_half<5, VT, XT>(A, x, ldx_, y, ldy, ycs, al, sg, be, st);
        return launch_spmv_half<6, VT, XT>(A, x, ldx_, y, ldy, ycs, al, sg, be, st);
    }

    const int64_t rows_per_warp = rowslot ? 32 / KW : 1;
    int64_t need = ((A->nrows + rows_per_warp - 1) / rows_per_warp * 32 + threads - 1) / threads;
    const int res = rowslot ? resident_blocks<k_spmm<KW, VT, XT, true>>(threads)
                            : resident_blocks<k_spmm<KW, VT, XT, false>>(threads);
    int64_t maxb = (int64_t)num_sms() * res;
    int64_t bx = need < maxb ? need : maxb;
    if (bx < 1) bx = 1;
    dim3 grid((unsigned)bx, (unsigned)((k + KW - 1) / KW));
    const int hs = (sg.x != 0.0 || sg.y != 0.0) ? 1 : 0;
    const int hb = (be.x != 0.0 || be.y != 0.0) ? 1 : 0;
    if (rowslot)
        k_spmm<KW, VT, XT, true><<<grid, threads, 0, st>>>(A->nrows, A->row_ptr, A->col,
                                                            reinterpret_cast<const VT*>(A->val), k,
                                                            reinterpret_cast<const XT*>(x), ldx_,
                                                            reinterpret_cast<XT*>(y), ldy, ycs, al, sg, be, hs, hb);
    else
        k_spmm<KW, VT, XT, false><<<grid, threads, 0, st>>>(A->nrows, A->row_ptr, A->col,
                                                             reinterpret_cast<const VT*>(A->val), k,
                                                             reinterpret_cast<const XT*>(x), ldx_,
                                                             reinterpret_cast<XT*>(y), ldy, ycs, al, sg, be, hs, hb);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <class VT, class XT>
static int launch_spmm_v(const edx_csr* A, int k, int kw, const void* x, int64_t ldx_, void* y,
                         int64_t ldy, int64_t ycs, double2 al, double2 sg, double2 be, cudaStream_t st) {
    switch (kw) {
    case 1: return launch_spmm_t<1, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 2: return launch_spmm_t<2, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 4: return launch_spmm_t<4, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 6: return launch_spmm_t<6, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 8: return launch_spmm_t<8, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 12: return launch_spmm_t<12, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 16: return launch_spmm_t<16, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    case 32: return launch_spmm_t<32, VT, XT>(A, k, x, ldx_, y, ldy, ycs, al, sg, be, st);
    }
    return fail(EDX_ERR_INVALID, "spmm: unsupported column group width %d", kw);
}

// columns per lane group: the smallest supported width >= k (k <= 32), else 32 with tiles
int auto_kw(int k) {
    static const int widths[] = {1, 2, 4, 6, 8, 12, 16, 32};
    for (int w : widths)
        if (w >= k) return w;
    return 32;
}

// power-of-two width for the element-wise recurrence kernels
int pow2_kw(int k) {
    int kw = 1;
    while (kw < k && kw < 32) kw <<= 1;
    return kw;
}

int check_csr(const edx_csr* A) {
    EDX_REQUIRE(A != nullptr, "NULL matrix");
    EDX_REQUIRE(A->nrows >= 0 && A->ncols >= 0 && A->nnz >= 0, "matrix with negative size");
    EDX_REQUIRE(A->nrows == 0 || A->row_ptr != nullptr, "matrix without row pointers");
    EDX_REQUIRE(A->nnz == 0 || (A->col != nullptr && A->val != nullptr), "matrix without entries");
    EDX_REQUIRE(A->val_type == EDX_C128 || A->val_type == EDX_C64, "matrix value type %d", A->val_type);
    return EDX_OK;
}

int spmm_dispatch(const edx_csr* A, int k, int vec_type, const void* x, int64_t ldx_, void* y, int64_t ldy,
                  int64_t ycs, double2 al, double2 sg, double2 be, int kw, cudaStream_t st) {
    if (kw <= 0) kw = auto_kw(k);
    if (A->val_type == EDX_C128) {
        EDX_REQUIRE(vec_type == EDX_C128, "spmm: a complex128 matrix needs complex128 vectors");
        return launch_spmm_v<double2, double2>(A, k, kw, x, ldx_, y, ldy, ycs, al, sg, be, st);
    }
    if (vec_type == EDX_C128) return launch_spmm_v<float2, double2>(A, k, kw, x, ldx_, y, ldy, ycs, al, sg, be, st);
    return launch_spmm_v<float2, float2>(A, k, kw, x, ldx_, y, ldy, ycs, al, sg, be, st);
}

// ---- the same product on the packed form ----------------------------------------------
// Value table in shared memory, diagonal term added with the store.  One column: warp per
// row with the next row's words prefetched; up to 16 columns per tile: one row per group of
// KW lanes; 32: warp per row.
template <int KW, bool WIDE>
__global__ void __launch_bounds__(256) k_spmm_packed(int64_t nrows, PackedView M, int k, const double2* __restrict__ X,
                                                     int64_t ldx_, double2* __restrict__ Y, int64_t ldy,
                                                     double2 alpha, double2 sigma, double2 beta, int has_sigma,
                                                     int has_beta) {
    extern __shared__ double2 sp_tab[];
    for (int i = threadIdx.x; i < M.nval; i += blockDim.x) sp_tab[i] = M.vals[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int c = lane % KW;
    const int col0 = blockIdx.y * KW;
    const int gc = col0 + c;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    auto store = [&](int64_t r, double2 acc) {
        const double2 xr = X[r * ldx_ + gc];
        const double2 a = fma_c(__ldg(M.diag + r), xr, acc);
        double yr = alpha.x * a.x - alpha.y * a.y;
        double yi = alpha.x * a.y + alpha.y * a.x;
        if (has_sigma) {
            yr += sigma.x * xr.x - sigma.y * xr.y;
            yi += sigma.x * xr.y + sigma.y * xr.x;
        }
        double2* yp = Y + r * ldy + gc;
        if (has_beta) {
            const double2 yv = *yp;
            yr += beta.x * yv.x - beta.y * yv.y;
            yi += beta.x * yv.y + beta.y * yv.x;
        }
        *yp = make_double2(yr, yi);
    };
    if constexpr (KW == 1) {  // one column: the next row's words load during this row
        spmv_rows_packed<WIDE>(warp0, nrows, nw, M, sp_tab, X, ldx_, col0, [&](int64_t r, double2 acc) {
            if (lane == 0) store(r, acc);
        });
    } else if constexpr (KW <= 16) {  // a few columns: each lane group walks a row of its own
        constexpr int SLOTS = 32 / KW;
        constexpr int U = 4;
        const int slot = lane / KW;
        const uint32_t vmask = WIDE ? 0u : (1u << M.vbits) - 1u;
        for (int64_t rb = warp0 * SLOTS; rb < nrows; rb += nw * SLOTS) {
            const int64_t r = rb + slot;
            const bool live = slot < SLOTS && r < nrows;
            const int64_t s = live ? __ldg(M.row_ptr + r) : 0, e = live ? __ldg(M.row_ptr + r + 1) : 0;
            double2 acc = make_double2(0.0, 0.0);
            for (int64_t j0 = s; j0 < e; j0 += U) {
                double2 v[U], xv[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int64_t j = j0 + u;
                    const bool ok = j < e;
                    int64_t cc = 0;
                    uint32_t q = 0;
                    if (ok)
                        pk_decode<WIDE>(__ldg(M.ent + j), WIDE ? (uint32_t)__ldg(M.vidx + j) : 0u, M.vbits, vmask, cc,
                                        q);
                    v[u] = ok ? sp_tab[q] : make_double2(0.0, 0.0);
                    xv[u] = (ok && gc < k) ? ldx(X + cc * ldx_ + gc) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) acc = fma_c(v[u], xv[u], acc);
            }
            if (live && gc < k) store(r, acc);
        }
    } else {
        for (int64_t r = warp0; r < nrows; r += nw) {
            const int64_t s = __ldg(M.row_ptr + r), e = __ldg(M.row_ptr + r + 1);
            double2 acc[1];
            row_times_x_packed<KW, 1, WIDE>(s, e, M.ent, M.vidx, M.vbits, sp_tab, X, ldx_, col0, k, acc);
            if (lane < KW && gc < k) store(r, acc[0]);
        }
    }
}

template <int KW, bool WIDE>
static int launch_spmm_packed_t(const PackedView& M, int64_t n, int k, const double2* x, int64_t ldx_, double2* y,
                                int64_t ldy, double2 al, double2 sg, double2 be, cudaStream_t st) {
    const int threads = 256;
    const size_t smem = (size_t)M.nval * sizeof(double2);
    static int cache[EDX_MAX_DEVICES] = {};
    int dev = 0;
    EDX_CUDA(cudaGetDevice(&dev));
    EDX_REQUIRE(dev >= 0 && dev < EDX_MAX_DEVICES, "edx_spmm_packed: device ordinal %d out of range", dev);
    if (cache[dev] == 0) {  // resident blocks with the largest table
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spmm_packed<KW, WIDE>, threads,
                                                          EDX_PACK_VALUES_MAX * sizeof(double2)) != cudaSuccess ||
            nb < 1)
            nb = 4;
        cache[dev] = nb;
    }
    const int64_t need = (n * 32 + threads - 1) / threads;
    const int64_t maxb = (int64_t)num_sms() * cache[dev];
    const int64_t bx = std::max<int64_t>(1, std::min(need, maxb));
    dim3 grid((unsigned)bx, (unsigned)((k + KW - 1) / KW));
    const int hs = (sg.x != 0.0 || sg.y != 0.0) ? 1 : 0;
    const int hb = (be.x != 0.0 || be.y != 0.0) ? 1 : 0;
    k_spmm_packed<KW, WIDE><<<grid, threads, smem, st>>>(n, M, k, x, ldx_, y, ldy, al, sg, be, hs, hb);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <bool WIDE>
static int launch_spmm_packed(const PackedView& M, int64_t n, int k, int kw, const double2* x, int64_t ldx_,
                              double2* y, int64_t ldy, double2 al, double2 sg, double2 be, cudaStream_t st) {
    switch (kw) {
    case 1: return launch_spmm_packed_t<1, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 2: return launch_spmm_packed_t<2, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 4: return launch_spmm_packed_t<4, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 6: return launch_spmm_packed_t<6, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 8: return launch_spmm_packed_t<8, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 12: return launch_spmm_packed_t<12, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 16: return launch_spmm_packed_t<16, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    case 32: return launch_spmm_packed_t<32, WIDE>(M, n, k, x, ldx_, y, ldy, al, sg, be, st);
    }
    return fail(EDX_ERR_INVALID, "edx_spmm_packed: unsupported column group width %d", kw);
}

}  // namespace edx

using namespace edx;

extern "C" int edx_spmm(const edx_csr* A, int k, int vec_type, const void* d_x, int64_t ldx_, void* d_y,
                        int64_t ldy, double alpha_re, double alpha_im, double sigma_re, double sigma_im,
                        double beta_re, double beta_im, int col_group, void* stream) {
    int rc = check_csr(A);
    if (rc) return rc;
    EDX_REQUIRE(k >= 1, "edx_spmm: k must be >= 1");
    EDX_REQUIRE(ldx_ >= k && ldy >= k, "edx_spmm: leading dimensions must be >= k");
    EDX_REQUIRE(d_x != nullptr && d_y != nullptr, "edx_spmm: NULL vectors");
    EDX_REQUIRE(vec_type == EDX_C128 || vec_type == EDX_C64, "edx_spmm: bad vec_type");
    if ((sigma_re != 0.0 || sigma_im != 0.0))
        EDX_REQUIRE(A->nrows == A->ncols, "edx_spmm: sigma needs a square matrix");
    EDX_REQUIRE(col_group == 0 || col_group == 1 || col_group == 2 || col_group == 4 || col_group == 6 ||
                    col_group == 8 || col_group == 12 || col_group == 16 || col_group == 32,
                "edx_spmm: column group width must be one of 1, 2, 4, 6, 8, 12, 16, 32");
    if (A->nrows == 0) return EDX_OK;
    return spmm_dispatch(A, k, vec_type, d_x, ldx_, d_y, ldy, 1, make_double2(alpha_re, alpha_im),
                         make_double2(sigma_re, sigma_im), make_double2(beta_re, beta_im), col_group,
                         as_stream(stream));
}

extern "C" int edx_spmm_packed(const edx_packed* P, int k, const double* d_x, int64_t ldx_, double* d_y, int64_t ldy,
                               double alpha_re, double alpha_im, double sigma_re, double sigma_im, double beta_re,
                               double beta_im, int col_group, void* stream) {
    EDX_REQUIRE(P != nullptr && P->nrows >= 0 && P->nnz >= 0, "edx_spmm_packed: bad matrix");
    EDX_REQUIRE(P->nrows == 0 || (P->row_ptr && P->diag), "edx_spmm_packed: matrix without row pointers");
    EDX_REQUIRE(P->nnz == 0 || (P->ent && P->vals && P->nval >= 1), "edx_spmm_packed: matrix without entries");
    EDX_REQUIRE(P->nval >= 0 && P->nval <= EDX_PACK_VALUES_MAX && P->vbits >= 0 && P->vbits <= 31,
                "edx_spmm_packed: bad value table");
    EDX_REQUIRE(P->vbits > 0 || P->nnz == 0 || P->vidx, "edx_spmm_packed: the wide form needs vidx");
    EDX_REQUIRE(k >= 1, "edx_spmm_packed: k must be >= 1");
    EDX_REQUIRE(ldx_ >= k && ldy >= k, "edx_spmm_packed: leading dimensions must be >= k");
    EDX_REQUIRE(d_x != nullptr && d_y != nullptr, "edx_spmm_packed: NULL vectors");
    EDX_REQUIRE(col_group == 0 || col_group == 1 || col_group == 2 || col_group == 4 || col_group == 6 ||
                    col_group == 8 || col_group == 12 || col_group == 16 || col_group == 32,
                "edx_spmm_packed: column group width must be one of 1, 2, 4, 6, 8, 12, 16, 32");
    if (P->nrows == 0) return EDX_OK;
    const int kw = col_group > 0 ? col_group : auto_kw(k);
    const PackedView M{P->row_ptr, P->ent, reinterpret_cast<const double2*>(P->vals),
                       reinterpret_cast<const double2*>(P->diag), P->vbits, P->nval, P->vidx};
    const double2 al = make_double2(alpha_re, alpha_im), sg = make_double2(sigma_re, sigma_im),
                  be = make_double2(beta_re, beta_im);
    const double2* x = reinterpret_cast<const double2*>(d_x);
    double2* y = reinterpret_cast<double2*>(d_y);
    if (P->vbits == 0) return launch_spmm_packed<true>(M, P->nrows, k, kw, x, ldx_, y, ldy, al, sg, be, as_stream(stream));
    return launch_spmm_packed<false>(M, P->nrows, k, kw, x, ldx_, y, ldy, al, sg, be, as_stream(stream));
}
