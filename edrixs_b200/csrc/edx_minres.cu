// edx_minres.cu -- one-RHS MINRES (K12, plain FP64 path), continued fraction (K13) and
// density matrix (K14).
#include <algorithm>
#include <mutex>

#include "edx_fock.cuh"
#include "edx_spmm.cuh"

namespace edx {

int check_csr(const edx_csr* A);
constexpr int MT = 256;

// ---- MINRES of src/linsys.f90:3-128 ----------------------------------------------------
// Device-resident scalar state; every kernel of iteration `it` is a no-op once
// stop_at >= 0 and it >= stop_at, so the host may launch ahead of the stopping test.
struct MinresState {
    double beta0, beta1, res;
    double2 alpha, gamma0, gamma1, sigma0, sigma1, eta, rho1, rho2, rho3, ge;
    int iter, stop_at;
    unsigned ticket[2];
};

__device__ __forceinline__ bool mr_skip(const MinresState* S, int it) {
    int s = *(volatile const int*)&S->stop_at;
    return s >= 0 && it >= s;
}

__device__ __forceinline__ bool mr_last(unsigned* ticket) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1u);
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[MT / 32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[q];
    __syncthreads();
    return s;  // valid in thread 0
}

__global__ void k_mr_scale(int64_t n, double2* __restrict__ v, MinresState* S, int it) {
    if (mr_skip(S, it)) return;
    const double b = S->beta0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 x = v[i];
        v[i] = make_double2(x.x / b, x.y / b);
    }
}

// tmp = op(A) v, alpha = <v, tmp>
template <class VT, int HALF>
__global__ void __launch_bounds__(MT) k_mr_apply(int64_t n, const int64_t* __restrict__ row_ptr,
                                                 const int32_t* __restrict__ col, const VT* __restrict__ val,
                                                 double2 aop, double2 sop, const double2* __restrict__ v,
                                                 double2* __restrict__ tmp, double* part, MinresState* S, int it) {
    if (mr_skip(S, it)) return;
    const int lane = threadIdx.x & 31;
    double pr = 0.0, pi = 0.0;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    auto epi = [&](int64_t r, double2 acc) {
        if ((lane & (HALF > 0 ? 15 : 31)) == 0) {  // the row's leading lane
            double2 vr = v[r];
            double2 t = cmul(aop, acc);
            if (sop.x != 0.0 || sop.y != 0.0) t = cadd(t, cmul(sop, vr));
            tmp[r] = t;
            pr += vr.x * t.x + vr.y * t.y;
            pi += vr.x * t.y - vr.y * t.x;
        }
    };
    if constexpr (HALF > 0)  // rows of <= ~100 entries: two per warp
        spmv_rows_half<HALF, VT, double2>(w0, nw, n, row_ptr, col, val, v, 1, 0, epi);
    else
        spmv_rows<VT, double2>(w0, n, nw, row_ptr, col, val, v, 1, 0, epi);
    double sr = block_sum(pr);
    double si = block_sum(pi);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sr;
        part[2 * blockIdx.x + 1] = si;
    }
    if (mr_last(&S->ticket[0])) {
        // every thread adds a fixed subset of the block partials, then a fixed-order tree
        double ar = 0.0, ai = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += MT) {
            ar += __ldcg(part + 2 * b);
            ai += __ldcg(part + 2 * b + 1);
        }
        ar = block_sum(ar);
        ai = block_sum(ai);
        if (threadIdx.x == 0) {
            S->alpha = make_double2(ar, ai);
            S->ticket[0] = 0u;
        }
    }
}

// v_prev = tmp - alpha v - beta0 v_prev; beta1 = |v_prev|; Givens scalars (linsys.f90:84-109)
__global__ void __launch_bounds__(MT) k_mr_orth(int64_t n, const double2* __restrict__ v, double2* __restrict__ vp,
                                                const double2* __restrict__ tmp, double* part, MinresState* S,
                                                int it, double tol, int maxit) {
    if (mr_skip(S, it)) return;
    const double2 a = S->alpha;
    const double b0 = S->beta0;
    double p = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 r = csub(csub(tmp[i], cmul(a, v[i])), cscale(vp[i], b0));
        vp[i] = r;
        p += r.x * r.x + r.y * r.y;
    }
    double s = block_sum(p);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (mr_last(&S->ticket[1])) {
        double t = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += MT) t += __ldcg(part + b);
        t = block_sum(t);
        if (threadIdx.x == 0) {
            const double beta1 = sqrt(t);
            MinresState q = *S;
            const double2 alpha = q.alpha;
            const double2 delta = csub(cmul(q.gamma0, alpha), cscale(cmul(q.gamma1, q.sigma0), q.beta0));
            const double2 rho1 = csqrt_(cadd(cmul(delta, delta), make_double2(beta1 * beta1, 0.0)));
            const double2 rho2 = cadd(cmul(q.sigma0, alpha), cscale(cmul(q.gamma1, q.gamma0), q.beta0));
            const double2 rho3 = cscale(q.sigma1, q.beta0);
            q.gamma1 = q.gamma0;
            q.sigma1 = q.sigma0;
            q.gamma0 = cdiv(delta, rho1);
            q.sigma0 = cdiv(make_double2(beta1, 0.0), rho1);
            q.ge = cmul(q.gamma0, q.eta);
            q.rho1 = rho1;
            q.rho2 = rho2;
            q.rho3 = rho3;
            q.beta1 = beta1;
            q.res = cabs_(q.sigma0) * q.res;
            q.eta = cmul(make_double2(-q.sigma0.x, -q.sigma0.y), q.eta);
            q.beta0 = beta1;
            q.iter = it + 1;
            if (!(q.res > tol && q.iter < maxit)) q.stop_at = it + 1;
            q.ticket[1] = 0u;
            q.ticket[0] = S->ticket[0];
            *S = q;
        }
    }
}

// w_prev = (v - rho3 w_prev - rho2 w_cur)/rho1; x += gamma0*eta*w_prev
__global__ void k_mr_update(int64_t n, const double2* __restrict__ v, double2* __restrict__ wp,
                            const double2* __restrict__ wc, double2* __restrict__ x, const MinresState* S, int it) {
    if (mr_skip(S, it)) return;
    const double2 r1 = S->rho1, r2 = S->rho2, r3 = S->rho3, ge = S->ge;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 t = cdiv(csub(csub(v[i], cmul(r3, wp[i])), cmul(r2, wc[i])), r1);
        wp[i] = t;
        x[i] = cadd(x[i], cmul(ge, t));
    }
}

__global__ void k_mr_init(int64_t n, const double2* __restrict__ b, double2* __restrict__ v,
                          double2* __restrict__ vp, double2* __restrict__ w0, double2* __restrict__ w1,
                          double2* __restrict__ x, double* part) {
    double p = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 q = b[i];
        v[i] = q;
        vp[i] = make_double2(0, 0);
        w0[i] = make_double2(0, 0);
        w1[i] = make_double2(0, 0);
        x[i] = make_double2(0, 0);
        p += q.x * q.x + q.y * q.y;
    }
    double s = block_sum(p);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_mr_init2(int nb, const double* part, MinresState* S, double tol, int maxit) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += part[b];
    MinresState q;
    q.beta0 = sqrt(t);
    q.beta1 = 0.0;
    q.res = q.beta0;
    q.alpha = make_double2(0, 0);
    q.gamma0 = make_double2(1, 0);
    q.gamma1 = make_double2(1, 0);
    q.sigma0 = make_double2(0, 0);
    q.sigma1 = make_double2(0, 0);
    q.eta = make_double2(q.beta0, 0);
    q.rho1 = q.rho2 = q.rho3 = q.ge = make_double2(0, 0);
    q.iter = 0;
    q.stop_at = (fabs(q.res) > tol && 0 < maxit) ? -1 : 0;
    q.ticket[0] = q.ticket[1] = 0u;
    *S = q;
}

// ---- continued fraction (plot_spectrum.py:41-61) -----------------------------------------
__global__ void k_cf(int nset, const int32_t* __restrict__ neff, const double* __restrict__ alpha,
                     const double* __restrict__ beta, int ld, const double* __restrict__ e0,
                     const double* __restrict__ norm, const double* __restrict__ weight, int ngrid,
                     const double* __restrict__ omega, const double* __restrict__ gamma, double* __restrict__ spec,
                     int per_set, int accumulate) {
    const double inv_pi = 1.0 / 3.141592653589793;
    const int64_t total = per_set ? (int64_t)nset * ngrid : (int64_t)ngrid;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int w = (int)(idx % ngrid);
        const int s0 = per_set ? (int)(idx / ngrid) : 0;
        const int s1 = per_set ? s0 + 1 : nset;
        double acc = 0.0;
        for (int s = s0; s < s1; ++s) {
            const double* a = alpha + (int64_t)s * ld;
            const double* b = beta + (int64_t)s * ld;
            const int ne = neff[s];
            const double xr = omega[w] + e0[s];
            const double xi = gamma[w];
            double2 t = make_double2(0.0, 0.0);
            for (int j = ne - 1; j >= 1; --j) {
                const double bb = b[j - 1] * b[j - 1];
                t = cdiv(make_double2(bb, 0.0), make_double2(xr - a[j] - t.x, xi - t.y));
            }
            t = cdiv(make_double2(1.0, 0.0), make_double2(xr - a[0] - t.x, xi - t.y));
            acc += -inv_pi * t.y * norm[s] * weight[s];
        }
        if (accumulate) spec[idx] += acc;
        else spec[idx] = acc;
    }
}

// ---- density matrix (ed_driver.f90:194-248) -------------------------------------------
// Each thread owns output entries (v, i, j) and walks one chunk of rows; partial sums per
// chunk are added in chunk order by k_denmat_sum.
__global__ void k_denmat(const uint64_t* __restrict__ fock, int64_t n, int search_norb, int search_nelec, int nv,
                         int nvec, const double2* __restrict__ vecs, int64_t rows_per_chunk,
                         double2* __restrict__ part) {
    extern __shared__ uint64_t tab[];
    if (search_norb > 0) binom_fill(tab, search_norb, search_nelec);
    __syncthreads();
    const int P = nvec * nv * nv;
    const int e = blockIdx.y * blockDim.x + threadIdx.x;
    if (e >= P) return;
    const int v = e / (nv * nv), i = (e / nv) % nv, j = e % nv;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_chunk;
    const int64_t r1 = min(n, r0 + rows_per_chunk);
    double2 acc = make_double2(0.0, 0.0);
    const int lo = min(i, j), hi = max(i, j);
    for (int64_t a = r0; a < r1; ++a) {
        const uint64_t s = fock[a];
        const double2 va = vecs[a * nvec + v];
        if (i == j) {
            if ((s >> i) & 1ull) acc = cadd(acc, make_double2(va.x * va.x + va.y * va.y, 0.0));
            continue;
        }
        if (cabs_(va) < 1e-10) continue;
        // hop: destroy lo, create hi (lo < hi), as the reference's i < j loop
        if (!((s >> lo) & 1ull)) continue;
        int par = below_parity(s, lo);
        uint64_t t = s & ~(1ull << lo);
        if ((t >> hi) & 1ull) continue;
        par ^= below_parity(t, hi);
        t |= 1ull << hi;
        int64_t b = (search_norb > 0) ? fock_rank(tab, search_norb, search_nelec, t) : fock_search(fock, n, t);
        if (b < 0) continue;
        const double2 vb = vecs[b * nvec + v];
        const double sg = par ? -1.0 : 1.0;
        // (lo, hi) gets conj(v_a) v_b sign; (hi, lo) gets conj(v_b) v_a sign
        double2 c = (i == lo) ? cconjmul(va, vb) : cconjmul(vb, va);
        acc = cadd(acc, cscale(c, sg));
    }
    part[(int64_t)blockIdx.x * P + e] = acc;
}

__global__ void k_denmat_sum(int nchunk, int P, const double2* __restrict__ part, double2* __restrict__ out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P) return;
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < nchunk; ++c) s = cadd(s, part[(int64_t)c * P + e]);
    out[e] = s;
}

static int mr_grid(int64_t n) {
    int64_t g = (int64_t)num_sms() * 4;
    int64_t need = (n + MT - 1) / MT;
    return (int)std::max<int64_t>(1, std::min(g, need));
}

static int denmat_chunks(int64_t n) {
    int64_t c = (int64_t)num_sms() * 2;
    int64_t need = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min(c, need));
}

}  // namespace edx

using namespace edx;

extern "C" int edx_minres_workspace(int64_t n, size_t* bytes) {
    EDX_REQUIRE(bytes != nullptr && n >= 1, "edx_minres_workspace: bad arguments");
    WorkspaceSize s;
    s.take<double2>((size_t)n * 5);
    s.take<double>((size_t)num_sms() * 16 + 16);  // two partials per block of k_mr_apply
    s.take<MinresState>(1);
    *bytes = s.bytes();
    return EDX_OK;
}

extern "C" int edx_minres(const edx_csr* A, double alpha_re, double alpha_im, double sigma_re, double sigma_im,
                          const double* d_b, double* d_x, double tol, int maxit, int* iters_out, double* res_out,
                          void* d_work, size_t work_bytes, void* stream) {
    int rc = check_csr(A);
    if (rc) return rc;
    EDX_REQUIRE(A->nrows == A->ncols && A->nrows >= 1, "edx_minres: matrix must be square and non-empty");
    EDX_REQUIRE(d_b && d_x, "edx_minres: NULL vectors");
    cudaStream_t st = as_stream(stream);
    const int64_t n = A->nrows;
    Workspace w(d_work, work_bytes);
    double2* vbuf = w.take<double2>((size_t)n * 5);
    double* part = w.take<double>((size_t)num_sms() * 16 + 16);
    MinresState* S = w.take<MinresState>(1);
    if (!S) return fail(EDX_ERR_WORKSPACE, "edx_minres: workspace too small");
    double2 *vc = vbuf, *vp = vbuf + n, *wc = vbuf + 2 * n, *wp = vbuf + 3 * n, *tmp = vbuf + 4 * n;
    double2* x = reinterpret_cast<double2*>(d_x);
    const int g = mr_grid(n);
    k_mr_init<<<g, MT, 0, st>>>(n, reinterpret_cast<const double2*>(d_b), vc, vp, wc, wp, x, part);
    EDX_CHECK_LAUNCH();
    k_mr_init2<<<1, 32, 0, st>>>(g, part, S, tol, maxit);
    EDX_CHECK_LAUNCH();
    const double2 aop = make_double2(alpha_re, alpha_im), sop = make_double2(sigma_re, sigma_im);
    // the SpMV runs as one wave of resident blocks (at most 8 per SM: the partials buffer)
    // two rows per warp for rows of <= 100 entries on average, with 5 entries per lane
    // prefetched up to 75 (see spmv_rows_half)
    const int half = A->nnz <= 100 * n ? (A->nnz <= 75 * n ? 5 : 6) : 0;
    int res = 4;
    if (A->val_type == EDX_C128)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res, half ? k_mr_apply<double2, 6> : k_mr_apply<double2, 0>, MT,
                                                      0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res, half ? k_mr_apply<float2, 6> : k_mr_apply<float2, 0>, MT,
                                                      0);
    res = std::max(1, std::min(res, 8));
    const int64_t warps = half ? (n + 1) / 2 : n;
    const int ga = (int)std::min<int64_t>((warps * 32 + MT - 1) / MT, (int64_t)num_sms() * res);
    const int poll = 8;
    for (int it = 0; it < maxit; ++it) {
        k_mr_scale<<<g, MT, 0, st>>>(n, vc, S, it);
        const double2* v2 = reinterpret_cast<const double2*>(A->val);
        const float2* v1 = reinterpret_cast<const float2*>(A->val);
        if (A->val_type == EDX_C128 && half == 5)
            k_mr_apply<double2, 5><<<ga, MT, 0, st>>>(n, A->row_ptr, A->col, v2, aop, sop, vc, tmp, part, S, it);
        else if (A->val_type == EDX_C128 && half == 6)
            k_mr_apply<double2, 6><<<ga, MT, 0, st>>>(n, A->row_ptr, A->col, v2, aop, sop, vc, tmp, part, S, it);
        else if (A->val_type == EDX_C128)
            k_mr_apply<double2, 0><<<ga, MT, 0, st>>>(n, A->row_ptr, A->col, v2, aop, sop, vc, tmp, part, S, it);
        else if (half == 5)
            k_mr_apply<float2, 5><<<ga, MT, 0, st>>>(n, A->row_ptr, A->col, v1, aop, sop, vc, tmp, part, S, it);
        else if (half == 6)
            k_mr_apply<float2, 6><<<ga, MT, 0, st>>>(n, A->row_ptr, A->col, v1, aop, sop, vc, tmp, part, S, it);
        else
            k_mr_apply<float2, 0><<<ga, MT, 0, st>>>(n, A->row_ptr, A->col, v1, aop, sop, vc, tmp, part, S, it);
        k_mr_orth<<<g, MT, 0, st>>>(n, vc, vp, tmp, part, S, it, tol, maxit);
        k_mr_update<<<g, MT, 0, st>>>(n, vc, wp, wc, x, S, it);
        EDX_CHECK_LAUNCH();
        std::swap(vc, vp);
        std::swap(wc, wp);
        if ((it + 1) % poll == 0) {
            int stop = -1;
            EDX_CUDA(cudaMemcpyAsync(&stop, &S->stop_at, sizeof(int), cudaMemcpyDeviceToHost, st));
            EDX_CUDA(cudaStreamSynchronize(st));
            if (stop >= 0) break;
        }
    }
    MinresState h;
    EDX_CUDA(cudaMemcpyAsync(&h, S, sizeof(MinresState), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    if (iters_out) *iters_out = h.iter;
    if (res_out) *res_out = h.res;
    return EDX_OK;
}

extern "C" int edx_cf_spectrum(int nset, const int32_t* d_neff, const double* d_alpha, const double* d_beta, int ld,
                               const double* d_e0, const double* d_norm, const double* d_weight, int ngrid,
                               const double* d_omega, const double* d_gamma, double* d_spec, int per_set,
                               int accumulate, void* stream) {
    EDX_REQUIRE(nset >= 1 && ngrid >= 1 && ld >= 1, "edx_cf_spectrum: bad sizes");
    EDX_REQUIRE(d_neff && d_alpha && d_beta && d_e0 && d_norm && d_weight && d_omega && d_gamma && d_spec,
                "edx_cf_spectrum: NULL argument");
    int64_t total = per_set ? (int64_t)nset * ngrid : ngrid;
    int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)num_sms() * 16);
    k_cf<<<blocks, 256, 0, as_stream(stream)>>>(nset, d_neff, d_alpha, d_beta, ld, d_e0, d_norm, d_weight, ngrid,
                                                 d_omega, d_gamma, d_spec, per_set, accumulate);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

extern "C" int edx_denmat_workspace(int64_t n, int nv, int nvec, size_t* bytes) {
    EDX_REQUIRE(bytes != nullptr && n >= 1 && nv >= 1 && nvec >= 1, "edx_denmat_workspace: bad arguments");
    WorkspaceSize s;
    s.take<double2>((size_t)denmat_chunks(n) * nvec * nv * nv);
    *bytes = s.bytes();
    return EDX_OK;
}

extern "C" int edx_denmat(const uint64_t* d_fock, int64_t n, int search_norb, int search_nelec, int nv, int nvec,
                          const double* d_vecs, double* d_out, void* d_work, size_t work_bytes, void* stream) {
    EDX_REQUIRE(d_fock && d_vecs && d_out && n >= 1 && nvec >= 1, "edx_denmat: bad arguments");
    EDX_REQUIRE(nv >= 1 && nv <= 63, "edx_denmat: nv must be 1..63");
    cudaStream_t st = as_stream(stream);
    const int nch = denmat_chunks(n);
    const int P = nvec * nv * nv;
    Workspace w(d_work, work_bytes);
    double2* part = w.take<double2>((size_t)nch * P);
    if (!part) return fail(EDX_ERR_WORKSPACE, "edx_denmat: workspace too small");
    const int64_t rpc = (n + nch - 1) / nch;
    dim3 grid(nch, (P + 255) / 256);
    size_t smem = search_norb > 0 ? binom_bytes(search_norb, search_nelec) : 0;
    k_denmat<<<grid, 256, smem, st>>>(d_fock, n, search_norb, search_nelec, nv, nvec,
                                      reinterpret_cast<const double2*>(d_vecs), rpc, part);
    EDX_CHECK_LAUNCH();
    k_denmat_sum<<<(P + 255) / 256, 256, 0, st>>>(nch, P, part, reinterpret_cast<double2*>(d_out));
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

// ---- density matrix with no allocation at all ---------------------------------------------
// Some hosts cannot give this library device memory: a host whose HBM is fully carved up
// by its own allocator before the solve (a serving process that has reserved its whole
// budget for resident Hamiltonians), or a thin foreign-language binding that only forwards
// the eigenvector buffers it was handed and has no CUDA allocator to make a workspace.
// edx_denmat_static keeps the per-chunk partial sums of k_denmat in a fixed array in the
// library's own device memory instead.
namespace edx {

static __device__ __align__(256) double2
    g_denmat_scratch[(size_t)EDX_DENMAT_STATIC_CHUNKS * EDX_DENMAT_STATIC_MAX_ENTRIES];

// Device address of g_denmat_scratch for the current device.  In host code the symbol's
// name is only a host-side stand-in, so the address is looked up with the device current.
// It is looked up on every call rather than cached: after cudaDeviceReset the library's
// device code is loaded again, possibly at another address, and a cached pointer would be
// stale.  Once the module is loaded the lookup is a cheap host-side query.
static int denmat_scratch_address(double2** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_denmat_scratch);
    if (e != cudaSuccess || p == nullptr)
        return fail(EDX_ERR_CUDA, "edx_denmat_static: cudaGetSymbolAddress of the scratch array failed: %s",
                    cudaGetErrorString(e));
    *out = static_cast<double2*>(p);
    return EDX_OK;
}

}  // namespace edx

extern "C" int edx_denmat_static(const uint64_t* d_fock, int64_t n, int search_norb, int search_nelec, int nv,
                                 int nvec, const double* d_vecs, double* d_out, void* stream) {
    EDX_REQUIRE(d_fock && d_vecs && d_out && n >= 1 && nvec >= 1, "edx_denmat_static: bad arguments");
    EDX_REQUIRE(nv >= 1 && nv <= 63, "edx_denmat_static: nv must be 1..63");
    const int64_t P = (int64_t)nvec * nv * nv;
    EDX_REQUIRE(P <= EDX_DENMAT_STATIC_MAX_ENTRIES,
                "edx_denmat_static: nvec*nv*nv = %lld exceeds the static scratch limit of %d entries "
                "(use edx_denmat with a workspace)",
                (long long)P, EDX_DENMAT_STATIC_MAX_ENTRIES);
    double2* part = nullptr;
    int rc = denmat_scratch_address(&part);
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    // every (chunk, entry) slot the sum below reads is written by this call's k_denmat, so
    // nothing in the scratch array has to be cleared first
    const int nch = std::min(denmat_chunks(n), EDX_DENMAT_STATIC_CHUNKS);
    const int64_t rpc = (n + nch - 1) / nch;
    dim3 grid(nch, (unsigned)((P + 255) / 256));
    size_t smem = search_norb > 0 ? binom_bytes(search_norb, search_nelec) : 0;
    k_denmat<<<grid, 256, smem, st>>>(d_fock, n, search_norb, search_nelec, nv, nvec,
                                      reinterpret_cast<const double2*>(d_vecs), rpc, part);
    EDX_CHECK_LAUNCH();
    k_denmat_sum<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(nch, (int)P, part, reinterpret_cast<double2*>(d_out));
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}
