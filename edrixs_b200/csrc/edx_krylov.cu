// edx_krylov.cu -- Lanczos / Krylov recurrences (K9), shifted MINRES (K12), continued
// fraction (K13) and density matrix (K14).
//
// All recurrences keep their scalars (alpha, beta, Givens rotations) in device memory so
// that an iteration is a fixed sequence of launches with no host round trip; the host only
// polls a "columns still active" counter every few iterations to stop launching.  Reductions
// are deterministic: every block writes per-column partial sums, and the last block to
// finish (atomic ticket) adds them in block order.
#include <cuda.h>

#include <algorithm>
#include <vector>

#include "edx_fock.cuh"
#include "edx_krylov.cuh"
#include "edx_spmm.cuh"

namespace edx {

int spmm_dispatch(const edx_csr* A, int k, int vec_type, const void* x, int64_t ldx_, void* y, int64_t ldy,
                  int64_t ycs, double2 al, double2 sg, double2 be, int kw, cudaStream_t st);
int check_csr(const edx_csr* A);
int auto_kw(int k);
int pow2_kw(int k);

constexpr int KT = 256;  // threads per block for the recurrence kernels

// Sum a per-thread value over threads of the block that share local column c (there are
// `groups` of them, laid out as sh[g*KW + c]); result written to part[bx*k + gc].
template <int KW, int NT = KT>
__device__ __forceinline__ void block_col_partial(double v, bool writer, int g, int groups, int c, int k,
                                                  double* part) {
    __shared__ double sh[NT];
    if (writer) sh[g * KW + c] = v;
    __syncthreads();
    if (threadIdx.x < KW) {
        double s = 0.0;
        for (int q = 0; q < groups; ++q) s += sh[q * KW + threadIdx.x];
        const int gcol = blockIdx.y * KW + threadIdx.x;
        if (gcol < k) part[(int64_t)blockIdx.x * k + gcol] = s;
    }
    __syncthreads();
}

// ---- K9a: W = A V_cur - beta_{i-1} V_prev (into V_prev), alpha partials ---------------
// Row mapping: interleaved (warp w of block b takes rows w + NW*(b + B*i)) or chunked (block
// b owns one contiguous range of rows).  Chunked keeps a block inside the contiguous row
// ranges that share the high (bath) bits of the Fock states, where the impurity-internal
// terms (Coulomb, spin-orbit, crystal field) land; their gathers then hit L1.
template <int KW, int TG, class VT, int NT>
__global__ void __launch_bounds__(NT) k_lanczos_apply(int64_t n, const int64_t* __restrict__ row_ptr,
                                                      const int32_t* __restrict__ col, const VT* __restrict__ val,
                                                      const double2* __restrict__ Vc, double2* __restrict__ Vp,
                                                      KrylovState S, int it, int chunked, int prefetch) {
    constexpr int NW = NT / 32;
    constexpr int BC = TG * KW;  // columns handled by this block
    const int64_t nnz = prefetch ? __ldg(row_ptr + n) : 0;
    __shared__ double sh[NW * BC];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = lane % KW;
    const int k = S.k;
    const int col0 = blockIdx.y * BC;
    double bprev[TG], scur[TG], apart[TG];
#pragma unroll
    for (int g = 0; g < TG; ++g) {
        const int gc = col0 + g * KW + c;
        bprev[g] = (gc < k && it > 0) ? S.beta[gc] * S.sprev[gc] : 0.0;
        scur[g] = gc < k ? S.scur[gc] : 0.0;
        apart[g] = 0.0;
    }
    int64_t r0, r1, rstep;
    if (chunked) {
        const int64_t per = (n + gridDim.x - 1) / gridDim.x;
        r0 = (int64_t)blockIdx.x * per + warp;
        r1 = min(n, (int64_t)(blockIdx.x + 1) * per);
        rstep = NW;
    } else {
        r0 = (int64_t)blockIdx.x * NW + warp;
        r1 = n;
        rstep = (int64_t)gridDim.x * NW;
    }
    for (int64_t r = r0; r < r1; r += rstep) {
        const int64_t s = __ldg(row_ptr + r), e = __ldg(row_ptr + r + 1);
        if (prefetch && lane == 0 && r + rstep < r1) {
            // bring this warp's next row (indices and values) into L2 while this one runs
            const int64_t sn = __ldg(row_ptr + r + rstep), en = __ldg(row_ptr + r + rstep + 1);
            prefetch_l2(col, sn * 4, en * 4, nnz * 4);
            prefetch_l2(val, sn * (int64_t)sizeof(VT), en * (int64_t)sizeof(VT), nnz * (int64_t)sizeof(VT));
        }
        double2 acc[TG];
        row_times_x_tiles<KW, TG, VT, double2>(s, e, col, val, Vc, k, col0, k, acc);
        if (lane < KW) {
#pragma unroll
            for (int g = 0; g < TG; ++g) {
                const int gc = col0 + g * KW + c;
                if (gc < k) {
                    const int64_t o = r * k + gc;
                    const double2 vp = Vp[o];
                    double2 w = make_double2(-bprev[g] * vp.x, -bprev[g] * vp.y);
                    w.x = w.x + scur[g] * acc[g].x;
                    w.y = w.y + scur[g] * acc[g].y;
                    Vp[o] = w;
                    const double2 vc = Vc[o];
                    apart[g] += vc.x * w.x + vc.y * w.y;  // Re(conj(U_i) w); alpha = scur * sum
                }
            }
        }
    }
    // per-block column partials: sh[warp][g*KW + c], summed over warps in order
    if (lane < KW) {
#pragma unroll
        for (int g = 0; g < TG; ++g) sh[warp * BC + g * KW + lane] = apart[g];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < BC; i += NT) {
        double s = 0.0;
        for (int w = 0; w < NW; ++w) s += sh[w * BC + i];
        if (col0 + i < k) S.part[(int64_t)blockIdx.x * k + col0 + i] = s;
    }
    __syncthreads();
    if (arrive_last(S.ticket)) {
        for (int j = threadIdx.x; j < k; j += NT) {
            const double a = S.scur[j] * sum_partials(S.part, gridDim.x, k, j);
            S.alpha[j] = a;
            if (S.active[j]) S.alpha_out[(int64_t)j * S.maxn + it] = a;
        }
        if (threadIdx.x == 0) *S.ticket = 0u;
    }
}

// ---- K9a on the packed form ---------------------------------------------------------------
// Same row mapping and epilogue as k_lanczos_apply.  The distinct values are copied to shared
// memory first; the diagonal term d_r v_r is added in the epilogue, where V_cur[r] is read
// anyway for alpha.
template <int KW, int TG, int NT, bool WIDE>
__global__ void __launch_bounds__(NT, 1024 / NT) k_lanczos_apply_packed(int64_t n, PackedView M, const double2* __restrict__ Vc,
                                                             double2* __restrict__ Vp, KrylovState S, int it,
                                                             int chunked) {
    constexpr int NW = NT / 32;
    constexpr int BC = TG * KW;
    extern __shared__ double2 pk_tab[];
    __shared__ double sh[NW * BC];
    for (int i = threadIdx.x; i < M.nval; i += NT) pk_tab[i] = M.vals[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = lane % KW;
    const int k = S.k;
    const int col0 = blockIdx.y * BC;
    double bprev[TG], scur[TG], apart[TG];
#pragma unroll
    for (int g = 0; g < TG; ++g) {
        const int gc = col0 + g * KW + c;
        bprev[g] = (gc < k && it > 0) ? S.beta[gc] * S.sprev[gc] : 0.0;
        scur[g] = gc < k ? S.scur[gc] : 0.0;
        apart[g] = 0.0;
    }
    int64_t r0, r1, rstep;
    if (chunked) {
        const int64_t per = (n + gridDim.x - 1) / gridDim.x;
        r0 = (int64_t)blockIdx.x * per + warp;
        r1 = min(n, (int64_t)(blockIdx.x + 1) * per);
        rstep = NW;
    } else {
        r0 = (int64_t)blockIdx.x * NW + warp;
        r1 = n;
        rstep = (int64_t)gridDim.x * NW;
    }
    for (int64_t r = r0; r < r1; r += rstep) {
        const int64_t s = __ldg(M.row_ptr + r), e = __ldg(M.row_ptr + r + 1);
        double2 acc[TG];
        row_times_x_packed<KW, TG, WIDE>(s, e, M.ent, M.vidx, M.vbits, pk_tab, Vc, k, col0, k, acc);
        if (lane < KW) {
            const double2 d = __ldg(M.diag + r);
#pragma unroll
            for (int g = 0; g < TG; ++g) {
                const int gc = col0 + g * KW + c;
                if (gc < k) {
                    const int64_t o = r * k + gc;
                    const double2 vc = Vc[o];
                    const double2 hv = fma_c(d, vc, acc[g]);
                    const double2 vp = Vp[o];
                    double2 w = make_double2(-bprev[g] * vp.x, -bprev[g] * vp.y);
                    w.x = w.x + scur[g] * hv.x;
                    w.y = w.y + scur[g] * hv.y;
                    Vp[o] = w;
                    apart[g] += vc.x * w.x + vc.y * w.y;  // Re(conj(U_i) w); alpha = scur * sum
                }
            }
        }
    }
    if (lane < KW) {
#pragma unroll
        for (int g = 0; g < TG; ++g) sh[warp * BC + g * KW + lane] = apart[g];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < BC; i += NT) {
        double s = 0.0;
        for (int w = 0; w < NW; ++w) s += sh[w * BC + i];
        if (col0 + i < k) S.part[(int64_t)blockIdx.x * k + col0 + i] = s;
    }
    __syncthreads();
    if (arrive_last(S.ticket)) {
        for (int j = threadIdx.x; j < k; j += NT) {
            const double a = S.scur[j] * sum_partials(S.part, gridDim.x, k, j);
            S.alpha[j] = a;
            if (S.active[j]) S.alpha_out[(int64_t)j * S.maxn + it] = a;
        }
        if (threadIdx.x == 0) *S.ticket = 0u;
    }
}

// ---- K9a on the packed form, one row per slot ------------------------------------------------
// For a few columns (k <= 16): each slot of KW lanes walks a row of its own, U entries at a
// time (the slot's lanes read the same word, then gather their own columns), so no
// cross-slot reduction runs per row and no lanes idle at the end of a row.  Rows of the
// block's warps are consecutive: warp w's slot q takes row (b*NW + w)*SLOTS + q of the
// sweep.  The epilogue and the alpha partials are those of k_lanczos_apply_packed.
template <int KW, int NT, bool WIDE>
__global__ void __launch_bounds__(NT, 1024 / NT) k_lanczos_apply_packed_rs(int64_t n, PackedView M,
                                                                            const double2* __restrict__ Vc,
                                                                            double2* __restrict__ Vp, KrylovState S,
                                                                            int it) {
    constexpr int NW = NT / 32;
    constexpr int SLOTS = 32 / KW;
    constexpr int U = 4;
    extern __shared__ double2 rs_tab[];
    __shared__ double sh[NW * KW];
    for (int i = threadIdx.x; i < M.nval; i += NT) rs_tab[i] = M.vals[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KW, c = lane % KW;
    const int k = S.k;
    const bool mine = slot < SLOTS && c < k;
    const uint32_t vmask = WIDE ? 0u : (1u << M.vbits) - 1u;
    const double bprev = (mine && it > 0) ? S.beta[c] * S.sprev[c] : 0.0;
    const double scur = mine ? S.scur[c] : 0.0;
    double apart = 0.0;
    const int64_t rstep = (int64_t)gridDim.x * NW * SLOTS;
    for (int64_t rb = ((int64_t)blockIdx.x * NW + warp) * SLOTS; rb < n; rb += rstep) {
        const int64_t r = rb + slot;
        const bool live = slot < SLOTS && r < n;
        const int64_t s = live ? __ldg(M.row_ptr + r) : 0, e = live ? __ldg(M.row_ptr + r + 1) : 0;
        double2 acc = make_double2(0.0, 0.0);
        for (int64_t j0 = s; j0 < e; j0 += U) {
            double2 v[U], x[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t j = j0 + u;
                const bool ok = j < e;
                int64_t cc = 0;
                uint32_t q = 0;
                if (ok) pk_decode<WIDE>(__ldg(M.ent + j), WIDE ? (uint32_t)__ldg(M.vidx + j) : 0u, M.vbits, vmask, cc, q);
                v[u] = ok ? rs_tab[q] : make_double2(0.0, 0.0);
                x[u] = (ok && c < k) ? ldx(Vc + cc * k + c) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) acc = fma_c(v[u], x[u], acc);
        }
        if (live && c < k) {
            const int64_t o = r * k + c;
            const double2 vc = Vc[o];
            const double2 hv = fma_c(__ldg(M.diag + r), vc, acc);
            const double2 vp = Vp[o];
            double2 w = make_double2(-bprev * vp.x, -bprev * vp.y);
            w.x = w.x + scur * hv.x;
            w.y = w.y + scur * hv.y;
            Vp[o] = w;
            apart += vc.x * w.x + vc.y * w.y;  // Re(conj(U_i) w); alpha = scur * sum
        }
    }
    // the slots' partials of each column, then the block's
    double tot = 0.0;
#pragma unroll
    for (int q = 0; q < SLOTS; ++q) tot += __shfl_sync(0xffffffffu, apart, q * KW + (lane % KW));
    if (lane < KW) sh[warp * KW + lane] = tot;
    __syncthreads();
    for (int i = threadIdx.x; i < KW; i += NT) {
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t += sh[w * KW + i];
        if (i < k) S.part[(int64_t)blockIdx.x * k + i] = t;
    }
    __syncthreads();
    if (arrive_last(S.ticket)) {
        for (int j = threadIdx.x; j < k; j += NT) {
            const double a = S.scur[j] * sum_partials(S.part, gridDim.x, k, j);
            S.alpha[j] = a;
            if (S.active[j]) S.alpha_out[(int64_t)j * S.maxn + it] = a;
        }
        if (threadIdx.x == 0) *S.ticket = 0u;
    }
}

// ---- K9a on the CSR, one row per slot (k <= KW <= 16) --------------------------------------
// As k_lanczos_apply_packed_rs, with the entries read from the CSR (row_times_x_slot).
template <int KW, class VT, int NT>
__global__ void __launch_bounds__(NT) k_lanczos_apply_rs(int64_t n, const int64_t* __restrict__ row_ptr,
                                                         const int32_t* __restrict__ col, const VT* __restrict__ val,
                                                         const double2* __restrict__ Vc, double2* __restrict__ Vp,
                                                         KrylovState S, int it) {
    constexpr int NW = NT / 32;
    constexpr int SLOTS = 32 / KW;
    __shared__ double sh[NW * KW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KW, c = lane % KW;
    const int k = S.k;
    const bool mine = slot < SLOTS && c < k;
    const double bprev = (mine && it > 0) ? S.beta[c] * S.sprev[c] : 0.0;
    const double scur = mine ? S.scur[c] : 0.0;
    double apart = 0.0;
    const int64_t rstep = (int64_t)gridDim.x * NW * SLOTS;
    for (int64_t rb = ((int64_t)blockIdx.x * NW + warp) * SLOTS; rb < n; rb += rstep) {
        const int64_t r = rb + slot;
        const bool live = slot < SLOTS && r < n;
        const int64_t s = live ? __ldg(row_ptr + r) : 0, e = live ? __ldg(row_ptr + r + 1) : 0;
        double2 acc;
        row_times_x_slot<KW, VT, double2>(s, e, col, val, Vc, k, c, c < k, acc);
        if (live && c < k) {
            const int64_t o = r * k + c;
            const double2 vp = Vp[o];
            double2 w = make_double2(-bprev * vp.x, -bprev * vp.y);
            w.x = w.x + scur * acc.x;
            w.y = w.y + scur * acc.y;
            Vp[o] = w;
            const double2 vc = Vc[o];
            apart += vc.x * w.x + vc.y * w.y;  // Re(conj(U_i) w); alpha = scur * sum
        }
    }
    double tot = 0.0;
#pragma unroll
    for (int q = 0; q < SLOTS; ++q) tot += __shfl_sync(0xffffffffu, apart, q * KW + (lane % KW));
    if (lane < KW) sh[warp * KW + lane] = tot;
    __syncthreads();
    for (int i = threadIdx.x; i < KW; i += NT) {
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t += sh[w * KW + i];
        if (i < k) S.part[(int64_t)blockIdx.x * k + i] = t;
    }
    __syncthreads();
    if (arrive_last(S.ticket)) {
        for (int j = threadIdx.x; j < k; j += NT) {
            const double a = S.scur[j] * sum_partials(S.part, gridDim.x, k, j);
            S.alpha[j] = a;
            if (S.active[j]) S.alpha_out[(int64_t)j * S.maxn + it] = a;
        }
        if (threadIdx.x == 0) *S.ticket = 0u;
    }
}

// ---- K9b: W -= alpha v_i, beta = |W|, next scales -----------------------------------------
// v_i = scur * U_i, so W -= (alpha * scur) U_i.  The last block of each column group (one
// ticket per group) finishes its columns: beta from the per-block partials (the group's
// threads each add a fixed subset of the blocks, then one thread adds the subsets in order),
// the reference's stopping rule (|beta| < 1e-10), the scales of the next step and its share
// of the active-column count.
template <int KW>
__global__ void __launch_bounds__(KT) k_lanczos_orth(int64_t n, const double2* __restrict__ Vc,
                                                     double2* __restrict__ Vp, KrylovState S,
                                                     unsigned* __restrict__ gticket, int it) {
    const int k = S.k;
    const int c = threadIdx.x % KW, g = threadIdx.x / KW, groups = KT / KW;
    const int gc = blockIdx.y * KW + c;
    const bool colok = gc < k;
    const double a = colok ? S.alpha[gc] * S.scur[gc] : 0.0;
    double part = 0.0;
    if (colok) {
        for (int64_t r = (int64_t)blockIdx.x * groups + g; r < n; r += (int64_t)gridDim.x * groups) {
            const int64_t o = r * k + gc;
            double2 w = Vp[o], v = Vc[o];
            w.x = w.x - a * v.x;
            w.y = w.y - a * v.y;
            Vp[o] = w;
            part += w.x * w.x + w.y * w.y;
        }
    }
    block_col_partial<KW>(part, true, g, groups, c, k, S.part);
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(gticket + blockIdx.y, 1u) == gridDim.x - 1u);
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double red[KT];
    double sub = 0.0;
    if (colok)
        for (int b = g; b < (int)gridDim.x; b += groups) sub += __ldcg(S.part + (int64_t)b * k + gc);
    red[threadIdx.x] = sub;
    __syncthreads();
    int act = 0;
    if (threadIdx.x < KW && colok) {
        double tot = 0.0;
        for (int q = 0; q < groups; ++q) tot += red[q * KW + c];
        const double b = sqrt(tot);
        const int j = gc;
        if (S.active[j]) {
            S.beta_out[(int64_t)j * S.maxn + it] = b;
            S.neff[j] = it + 1;
            if (fabs(b) < 1e-10) S.active[j] = 0;
        }
        S.beta[j] = b;
        S.sprev[j] = S.scur[j];
        S.scur[j] = S.active[j] ? 1.0 / b : 0.0;
        act = S.active[j];
    }
    if (threadIdx.x < 32) {
        act = __reduce_add_sync(0xffffffffu, act);
        if (threadIdx.x == 0) {
            if (act) atomicAdd(S.n_active, act);
            gticket[blockIdx.y] = 0u;
        }
    }
}

// projections of U_i scaled to v_i = scur * U_i: out[(j*maxn + i)*m + r] *= scur[j]
__global__ void k_proj_scale(int64_t m, int k, int64_t maxn, int i, double2* __restrict__ out,
                             const double* __restrict__ scur) {
    const int64_t total = m * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / m);
        const int64_t r = e - (int64_t)j * m;
        double2* p = out + ((int64_t)j * maxn + i) * m + r;
        const double f = scur[j];
        double2 v = *p;
        *p = make_double2(v.x * f, v.y * f);
    }
}

// streaming projections: out[r * ld + s] += sum_{b < nb} coef[s * maxn + i0 + b] *
// win[(c * B + b) * m + r], c = acc_col[s]; win holds the last nb projected vectors
__global__ void k_proj_accum(int64_t m, int B, int nb, int i0, int64_t maxn, int nacc,
                             const int32_t* __restrict__ acc_col, const double2* __restrict__ coef,
                             const double2* __restrict__ win, double2* __restrict__ out, int64_t ld) {
    const int64_t total = m * nacc;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / nacc;
        const int s = (int)(e - r * nacc);
        const double2* w = win + (int64_t)acc_col[s] * B * m + r;
        const double2* cf = coef + (int64_t)s * maxn + i0;
        double2* o = out + r * ld + s;
        double2 a = *o;
        for (int b = 0; b < nb; ++b) a = fma_c(cf[b], w[(int64_t)b * m], a);
        *o = a;
    }
}

// ---- start vectors: norm and normalisation --------------------------------------------
template <int KW>
__global__ void __launch_bounds__(KT) k_colnorm(int64_t n, const double2* __restrict__ V0, int64_t ld0,
                                                KrylovState S) {
    const int k = S.k;
    const int c = threadIdx.x % KW, g = threadIdx.x / KW, groups = KT / KW;
    const int gc = blockIdx.y * KW + c;
    double part = 0.0;
    if (gc < k)
        for (int64_t r = (int64_t)blockIdx.x * groups + g; r < n; r += (int64_t)gridDim.x * groups) {
            double2 v = V0[r * ld0 + gc];
            part += v.x * v.x + v.y * v.y;
        }
    block_col_partial<KW>(part, true, g, groups, c, k, S.part);
    if (arrive_last(S.ticket + 2)) {
        for (int j = threadIdx.x; j < k; j += KT) {
            double s = sum_partials(S.part, gridDim.x, k, j);
            S.alpha[j] = s;  // <v0|v0>, handed to the host-side norm output
            S.beta[j] = sqrt(s);
            S.active[j] = 1;
            S.neff[j] = 0;
            S.scur[j] = 1.0;  // v_0 is stored normalised
            S.sprev[j] = 0.0;
        }
        if (threadIdx.x == 0) S.ticket[2] = 0u;
    }
}

__global__ void k_start(int64_t n, int k, const double2* __restrict__ V0, int64_t ld0, double2* __restrict__ Vc,
                        double2* __restrict__ Vp, const double* __restrict__ s) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k;
        const int c = (int)(e - r * k);
        double2 v = V0[r * ld0 + c];
        const double d = s[c];
        // a zero start vector stays zero (its recurrence stops after one step with norm 0),
        // where v / |v| would fill the column with NaN
        Vc[e] = d > 0.0 ? make_double2(v.x / d, v.y / d) : make_double2(0.0, 0.0);
        Vp[e] = make_double2(0.0, 0.0);
    }
}

// ---- K12: per-shift MINRES recurrences in the Lanczos basis ----------------------------
struct ShiftState {
    double2 gamma0, gamma1, sigma0, sigma1, eta;
    double beta0, res;
    int frozen, iters;
};

__global__ void k_shift_init(int nshift, const int32_t* __restrict__ scol, const double* __restrict__ norm2,
                             ShiftState* __restrict__ st, double tol, int maxit) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshift) return;
    const double b0 = sqrt(norm2[scol[s]]);
    ShiftState q;
    q.gamma0 = make_double2(1.0, 0.0);
    q.gamma1 = make_double2(1.0, 0.0);
    q.sigma0 = make_double2(0.0, 0.0);
    q.sigma1 = make_double2(0.0, 0.0);
    q.eta = make_double2(b0, 0.0);
    q.beta0 = b0;
    q.res = b0;
    q.iters = 0;
    q.frozen = !(fabs(b0) > tol && 0 < maxit);
    st[s] = q;
}

// one warp per shift; lanes share the scalar work and split the coefficient vectors
__global__ void k_shift_step(int nshift, const int32_t* __restrict__ scol, const double2* __restrict__ sz,
                             ShiftState* __restrict__ st, double2* __restrict__ wbuf, double2* __restrict__ y,
                             KrylovState S, int it, double tol, int maxit, int* __restrict__ n_open) {
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= nshift) return;
    ShiftState q = st[s];
    if (q.frozen) return;
    const int c = scol[s];
    if (S.neff[c] != it + 1) {  // the column's recurrence stopped before this iteration
        if (lane == 0) {
            q.frozen = 1;
            st[s] = q;
        }
        return;
    }
    const int64_t m = S.maxn;
    const double a_h = S.alpha_out[(int64_t)c * m + it];
    const double beta1 = S.beta_out[(int64_t)c * m + it];
    const double2 z = sz[s];
    const double2 alpha = make_double2(z.x - a_h, z.y);
    // linsys.f90:92-101
    const double2 delta = csub(cmul(q.gamma0, alpha), cscale(cmul(q.gamma1, q.sigma0), q.beta0));
    const double2 rho1 = csqrt_(cadd(cmul(delta, delta), make_double2(beta1 * beta1, 0.0)));
    const double2 rho2 = cadd(cmul(q.sigma0, alpha), cscale(cmul(q.gamma1, q.gamma0), q.beta0));
    const double2 rho3 = cscale(q.sigma1, q.beta0);
    q.gamma1 = q.gamma0;
    q.sigma1 = q.sigma0;
    q.gamma0 = cdiv(delta, rho1);
    q.sigma0 = cdiv(make_double2(beta1, 0.0), rho1);
    const double2 ge = cmul(q.gamma0, q.eta);
    // coefficient vectors: prev slot holds w_{it-2}, curr slot w_{it-1}; v_it = (-1)^it u_it
    double2* wprev = wbuf + ((int64_t)s * 2 + (it & 1)) * m;
    const double2* wcurr = wbuf + ((int64_t)s * 2 + ((it + 1) & 1)) * m;
    double2* ys = y + (int64_t)s * m;
    const double sgn = (it & 1) ? -1.0 : 1.0;
    for (int j = lane; j <= it; j += 32) {
        double2 v = make_double2(j == it ? sgn : 0.0, 0.0);
        double2 t = csub(csub(v, cmul(rho3, wprev[j])), cmul(rho2, wcurr[j]));
        double2 wn = cdiv(t, rho1);
        wprev[j] = wn;
        ys[j] = cadd(ys[j], cmul(ge, wn));
    }
    if (lane == 0) {
        q.res = cabs_(q.sigma0) * q.res;
        q.eta = cmul(make_double2(-q.sigma0.x, -q.sigma0.y), q.eta);
        q.beta0 = beta1;
        q.iters = it + 1;
        q.frozen = !(q.res > tol && q.iters < maxit);
        st[s] = q;
        if (!q.frozen) atomicAdd(n_open, 1);
    }
}

__global__ void k_shift_final(int nshift, const ShiftState* __restrict__ st, int32_t* iters, double* res) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshift) return;
    if (iters) iters[s] = st[s].iters;
    if (res) res[s] = st[s].res;
}

// launch shape of the fused apply kernel (chosen by the caller's autotuner, or defaults)
struct ApplyCfg {
    int kw;         // columns per lane group
    int tg;         // column tiles per block (1, 2, 4; >1 only for kw 16 / 32)
    int threads;    // 256 or 1024
    int gx;         // blocks along the rows
    int chunked;    // contiguous row ranges per block
    int prefetch;   // bulk-prefetch each warp's next row into L2
    int rowslot;    // packed form, k <= kw <= 16: one row per slot (k_lanczos_apply_packed_rs)
};

template <int KW, int TG, class VT, int NT>
static int launch_apply_nt(const edx_csr* A, const double2* Vc, double2* Vp, const KrylovState& S, int it,
                           const ApplyCfg& cfg, cudaStream_t st) {
    auto kern = k_lanczos_apply<KW, TG, VT, NT>;
    static bool carve_set = false;  // prefer L1 over shared memory: gathers are served from L1
    if (!carve_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        carve_set = true;
    }
    const int ntiles = (S.k + KW - 1) / KW;
    dim3 grid(cfg.gx, (ntiles + TG - 1) / TG);
    kern<<<grid, NT, 0, st>>>(A->nrows, A->row_ptr, A->col, reinterpret_cast<const VT*>(A->val), Vc, Vp, S, it,
                              cfg.chunked, cfg.prefetch);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <int KW, int TG, class VT>
static int launch_apply(const edx_csr* A, const double2* Vc, double2* Vp, const KrylovState& S, int it,
                        const ApplyCfg& cfg, cudaStream_t st) {
    if (cfg.threads == 1024) return launch_apply_nt<KW, TG, VT, 1024>(A, Vc, Vp, S, it, cfg, st);
    return launch_apply_nt<KW, TG, VT, 256>(A, Vc, Vp, S, it, cfg, st);
}

template <int KW, class VT>
static int launch_apply_tg(const edx_csr* A, const double2* Vc, double2* Vp, const KrylovState& S, int it,
                           const ApplyCfg& cfg, cudaStream_t st) {
    switch (cfg.tg) {
    case 2: return launch_apply<KW, 2, VT>(A, Vc, Vp, S, it, cfg, st);
    case 4: return launch_apply<KW, 4, VT>(A, Vc, Vp, S, it, cfg, st);
    default: return launch_apply<KW, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    }
}

template <int KW, class VT>
static int launch_apply_rs(const edx_csr* A, const double2* Vc, double2* Vp, const KrylovState& S, int it,
                           const ApplyCfg& cfg, cudaStream_t st) {
    const VT* v = reinterpret_cast<const VT*>(A->val);
    if (cfg.threads == 1024)
        k_lanczos_apply_rs<KW, VT, 1024><<<cfg.gx, 1024, 0, st>>>(A->nrows, A->row_ptr, A->col, v, Vc, Vp, S, it);
    else
        k_lanczos_apply_rs<KW, VT, 256><<<cfg.gx, 256, 0, st>>>(A->nrows, A->row_ptr, A->col, v, Vc, Vp, S, it);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <class VT>
static int apply_v(const edx_csr* A, const double2* Vc, double2* Vp, const KrylovState& S, int it,
                   const ApplyCfg& cfg, cudaStream_t st) {
    if (cfg.rowslot) {
        switch (cfg.kw) {
        case 1: return launch_apply_rs<1, VT>(A, Vc, Vp, S, it, cfg, st);
        case 2: return launch_apply_rs<2, VT>(A, Vc, Vp, S, it, cfg, st);
        case 4: return launch_apply_rs<4, VT>(A, Vc, Vp, S, it, cfg, st);
        case 6: return launch_apply_rs<6, VT>(A, Vc, Vp, S, it, cfg, st);
        case 8: return launch_apply_rs<8, VT>(A, Vc, Vp, S, it, cfg, st);
        case 12: return launch_apply_rs<12, VT>(A, Vc, Vp, S, it, cfg, st);
        case 16: return launch_apply_rs<16, VT>(A, Vc, Vp, S, it, cfg, st);
        }
        return fail(EDX_ERR_INVALID, "krylov: one row per slot needs a column group of at most 16");
    }
    switch (cfg.kw) {
    case 1: return launch_apply<1, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    case 2: return launch_apply<2, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    case 4: return launch_apply<4, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    case 6: return launch_apply<6, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    case 8: return launch_apply<8, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    case 12: return launch_apply<12, 1, VT>(A, Vc, Vp, S, it, cfg, st);
    case 16: return launch_apply_tg<16, VT>(A, Vc, Vp, S, it, cfg, st);
    case 32: return launch_apply_tg<32, VT>(A, Vc, Vp, S, it, cfg, st);
    }
    return fail(EDX_ERR_INVALID, "krylov: bad column group %d", cfg.kw);
}

template <int KW, int TG, int NT, bool WIDE>
static int launch_packed_nt(int64_t n, const PackedView& M, const double2* Vc, double2* Vp, const KrylovState& S,
                            int it, const ApplyCfg& cfg, cudaStream_t st) {
    auto kern = k_lanczos_apply_packed<KW, TG, NT, WIDE>;
    static bool attr_set[EDX_MAX_DEVICES] = {};
    int dev = 0;
    EDX_CUDA(cudaGetDevice(&dev));
    EDX_REQUIRE(dev >= 0 && dev < EDX_MAX_DEVICES, "edx_krylov: device ordinal %d out of range", dev);
    if (!attr_set[dev]) {
        EDX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(EDX_PACK_VALUES_MAX * sizeof(double2))));
        attr_set[dev] = true;
    }
    const int ntiles = (S.k + KW - 1) / KW;
    dim3 grid(cfg.gx, (ntiles + TG - 1) / TG);
    kern<<<grid, NT, (size_t)M.nval * sizeof(double2), st>>>(n, M, Vc, Vp, S, it, cfg.chunked);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <int KW, int TG>
static int launch_packed(int64_t n, const PackedView& M, const double2* Vc, double2* Vp, const KrylovState& S,
                         int it, const ApplyCfg& cfg, cudaStream_t st) {
    if (M.vbits == 0) {
        if (cfg.threads == 1024) return launch_packed_nt<KW, TG, 1024, true>(n, M, Vc, Vp, S, it, cfg, st);
        return launch_packed_nt<KW, TG, 256, true>(n, M, Vc, Vp, S, it, cfg, st);
    }
    if (cfg.threads == 1024) return launch_packed_nt<KW, TG, 1024, false>(n, M, Vc, Vp, S, it, cfg, st);
    return launch_packed_nt<KW, TG, 256, false>(n, M, Vc, Vp, S, it, cfg, st);
}

template <int KW, int NT, bool WIDE>
static int launch_packed_rs_nt(int64_t n, const PackedView& M, const double2* Vc, double2* Vp, const KrylovState& S,
                               int it, const ApplyCfg& cfg, cudaStream_t st) {
    auto kern = k_lanczos_apply_packed_rs<KW, NT, WIDE>;
    static bool attr_set[EDX_MAX_DEVICES] = {};
    int dev = 0;
    EDX_CUDA(cudaGetDevice(&dev));
    EDX_REQUIRE(dev >= 0 && dev < EDX_MAX_DEVICES, "edx_krylov: device ordinal %d out of range", dev);
    if (!attr_set[dev]) {
        EDX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(EDX_PACK_VALUES_MAX * sizeof(double2))));
        attr_set[dev] = true;
    }
    kern<<<cfg.gx, NT, (size_t)M.nval * sizeof(double2), st>>>(n, M, Vc, Vp, S, it);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <int KW>
static int launch_packed_rs(int64_t n, const PackedView& M, const double2* Vc, double2* Vp, const KrylovState& S,
                            int it, const ApplyCfg& cfg, cudaStream_t st) {
    if (M.vbits == 0) {
        if (cfg.threads == 1024) return launch_packed_rs_nt<KW, 1024, true>(n, M, Vc, Vp, S, it, cfg, st);
        return launch_packed_rs_nt<KW, 256, true>(n, M, Vc, Vp, S, it, cfg, st);
    }
    if (cfg.threads == 1024) return launch_packed_rs_nt<KW, 1024, false>(n, M, Vc, Vp, S, it, cfg, st);
    return launch_packed_rs_nt<KW, 256, false>(n, M, Vc, Vp, S, it, cfg, st);
}

static int apply_packed(const edx_packed* P, const double2* Vc, double2* Vp, const KrylovState& S, int it,
                        const ApplyCfg& cfg, cudaStream_t st) {
    const PackedView M{P->row_ptr, P->ent, reinterpret_cast<const double2*>(P->vals),
                       reinterpret_cast<const double2*>(P->diag), P->vbits, P->nval, P->vidx};
    const int64_t n = P->nrows;
    if (cfg.rowslot) {
        switch (cfg.kw) {
        case 1: return launch_packed_rs<1>(n, M, Vc, Vp, S, it, cfg, st);
        case 2: return launch_packed_rs<2>(n, M, Vc, Vp, S, it, cfg, st);
        case 4: return launch_packed_rs<4>(n, M, Vc, Vp, S, it, cfg, st);
        case 6: return launch_packed_rs<6>(n, M, Vc, Vp, S, it, cfg, st);
        case 8: return launch_packed_rs<8>(n, M, Vc, Vp, S, it, cfg, st);
        case 12: return launch_packed_rs<12>(n, M, Vc, Vp, S, it, cfg, st);
        case 16: return launch_packed_rs<16>(n, M, Vc, Vp, S, it, cfg, st);
        }
        return fail(EDX_ERR_INVALID, "krylov: one row per slot needs a column group of at most 16");
    }
    switch (cfg.kw) {
    case 1: return launch_packed<1, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 2: return launch_packed<2, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 4: return launch_packed<4, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 6: return launch_packed<6, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 8: return launch_packed<8, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 12: return launch_packed<12, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 16:
        if (cfg.tg == 4) return launch_packed<16, 4>(n, M, Vc, Vp, S, it, cfg, st);
        if (cfg.tg == 2) return launch_packed<16, 2>(n, M, Vc, Vp, S, it, cfg, st);
        return launch_packed<16, 1>(n, M, Vc, Vp, S, it, cfg, st);
    case 32:
        if (cfg.tg == 4) return launch_packed<32, 4>(n, M, Vc, Vp, S, it, cfg, st);
        if (cfg.tg == 2) return launch_packed<32, 2>(n, M, Vc, Vp, S, it, cfg, st);
        return launch_packed<32, 1>(n, M, Vc, Vp, S, it, cfg, st);
    }
    return fail(EDX_ERR_INVALID, "krylov: bad column group %d", cfg.kw);
}

#define EDX_KW_SWITCH(kw, KERNEL, GRID, ...)                                                  \
    switch (kw) {                                                                              \
    case 1: KERNEL<1><<<GRID, KT, 0, st>>>(__VA_ARGS__); break;                               \
    case 2: KERNEL<2><<<GRID, KT, 0, st>>>(__VA_ARGS__); break;                               \
    case 4: KERNEL<4><<<GRID, KT, 0, st>>>(__VA_ARGS__); break;                               \
    case 8: KERNEL<8><<<GRID, KT, 0, st>>>(__VA_ARGS__); break;                               \
    case 16: KERNEL<16><<<GRID, KT, 0, st>>>(__VA_ARGS__); break;                             \
    default: KERNEL<32><<<GRID, KT, 0, st>>>(__VA_ARGS__); break;                             \
    }

struct KrylovWs {
    double2 *Vc, *Vp;
    double *alpha, *beta, *part, *scur, *sprev;
    int *active, *n_active, *n_open, *kron_err;
    unsigned* ticket;
    unsigned* kticket;  // one per column tile of the slab product
    unsigned* gticket;  // one per 32 columns (per-group finish of the orthogonalisation)
    ShiftState* sst;
    double2* wbuf;
};

static int reduce_grid(int64_t n) {
    int64_t g = (int64_t)num_sms() * 4;
    int64_t need = (n + 63) / 64;
    if (need < g) g = need;
    if (g < 1) g = 1;
    return (int)g;
}

template <class WS>
static void krylov_layout(WS& w, int64_t n, int k, int nshift, int maxn, int gx, KrylovWs* out) {
    auto Vc = w.template take<double2>((size_t)(n * k));
    auto Vp = w.template take<double2>((size_t)(n * k));
    auto al = w.template take<double>((size_t)k);
    auto be = w.template take<double>((size_t)k);
    auto sc = w.template take<double>((size_t)k);
    auto sp = w.template take<double>((size_t)k);
    auto pa = w.template take<double>((size_t)gx * k);
    auto ac = w.template take<int>((size_t)k);
    auto na = w.template take<int>(3);
    auto tk = w.template take<unsigned>(4);
    auto kt = w.template take<unsigned>((size_t)k);
    auto gt = w.template take<unsigned>((size_t)(k + 31) / 32);
    auto ss = w.template take<ShiftState>((size_t)(nshift > 0 ? nshift : 1));
    auto wb = w.template take<double2>((size_t)(nshift > 0 ? 2 * (size_t)nshift * maxn : 1));
    if (out) {
        out->Vc = Vc;
        out->Vp = Vp;
        out->alpha = al;
        out->beta = be;
        out->scur = sc;
        out->sprev = sp;
        out->part = pa;
        out->active = ac;
        out->n_active = na;
        out->n_open = na + 1;
        out->kron_err = na + 2;
        out->ticket = tk;
        out->kticket = kt;
        out->gticket = gt;
        out->sst = ss;
        out->wbuf = wb;
    }
}

// WorkspaceSize::take returns void; wrap it so krylov_layout can use one template
struct SizeOnly {
    WorkspaceSize s;
    template <class T>
    T* take(size_t c) {
        s.take<T>(c);
        return nullptr;
    }
};

}  // namespace edx

using namespace edx;

extern "C" int edx_krylov_workspace(int64_t n, int k, const edx_krylov_opts* opts, int maxn, size_t* bytes) {
    EDX_REQUIRE(bytes != nullptr && n >= 1 && k >= 1 && maxn >= 1, "edx_krylov_workspace: bad arguments");
    SizeOnly s;
    int gx = num_sms() * 8;  // largest grid any kernel here uses
    if (opts && opts->apply_kron) {
        int rc = kron_check(opts->apply_kron);
        if (rc) return rc;
        gx = std::max(gx, kron_grid_x(opts->apply_kron, k, kron_col_group(k, opts->apply_col_group),
                                      opts->apply_blocks_per_sm));
    }
    krylov_layout(s, n, k, opts ? opts->nshift : 0, maxn, gx, nullptr);
    *bytes = s.s.bytes();
    return EDX_OK;
}

extern "C" int edx_krylov(const edx_csr* A, int k, const double* d_v0, int maxn, double* d_alpha, double* d_beta,
                          double* d_norm, int32_t* d_neff, const edx_krylov_opts* opts, void* d_work,
                          size_t work_bytes, void* stream) {
    int rc = check_csr(A);
    if (rc) return rc;
    EDX_REQUIRE(A->nrows == A->ncols && A->nrows >= 1, "edx_krylov: matrix must be square and non-empty");
    EDX_REQUIRE(k >= 1 && maxn >= 1 && d_v0 && d_alpha && d_beta && d_norm && d_neff,
                "edx_krylov: bad arguments");
    const int nshift = opts ? opts->nshift : 0;
    const int nproj = opts ? opts->nproj : 0;
    const int64_t ld0 = (opts && opts->v0_ld > 0) ? opts->v0_ld : k;
    EDX_REQUIRE(ld0 >= k, "edx_krylov: v0_ld must be >= k");
    if (nshift > 0)
        EDX_REQUIRE(opts->shift_col && opts->shift_z && opts->shift_y, "edx_krylov: shift arrays missing");
    for (int p = 0; p < nproj; ++p) {
        EDX_REQUIRE(opts->proj && opts->proj_out && opts->proj_out[p], "edx_krylov: projection %d missing", p);
        rc = check_csr(&opts->proj[p]);
        if (rc) return rc;
        EDX_REQUIRE(opts->proj[p].ncols == A->nrows, "edx_krylov: projection %d has wrong width", p);
    }
    const int win = (opts && nproj > 0 && opts->proj_window > 0) ? opts->proj_window : 0;
    if (win) {
        EDX_REQUIRE(opts->nacc >= 1 && opts->acc_col && opts->acc_coef && opts->acc_out && opts->acc_ld >= opts->nacc,
                    "edx_krylov: streaming projections need nacc, acc_col, acc_coef, acc_out and acc_ld >= nacc");
        for (int p = 0; p < nproj; ++p)
            EDX_REQUIRE(opts->acc_out[p], "edx_krylov: accumulator %d missing", p);
    }
    cudaStream_t st = as_stream(stream);
    const int64_t n = A->nrows;
    ApplyCfg cfg;
    cfg.kw = (opts && opts->apply_col_group > 0) ? opts->apply_col_group : auto_kw(k);
    cfg.threads = (opts && opts->apply_threads > 0) ? opts->apply_threads : 1024;
    const int bps = (opts && opts->apply_blocks_per_sm > 0) ? opts->apply_blocks_per_sm : 1;
    cfg.chunked = (opts && opts->apply_chunked > 0) ? 1 : 0;
    cfg.prefetch = (opts && opts->apply_prefetch > 0) ? 1 : 0;
    cfg.rowslot = (opts && opts->apply_rowslot > 0) ? 1 : 0;
    const int ntiles = (k + cfg.kw - 1) / cfg.kw;
    cfg.tg = (opts && opts->apply_tiles > 0) ? opts->apply_tiles : (ntiles >= 4 ? 4 : (ntiles >= 2 ? 2 : 1));
    if (cfg.kw < 16) cfg.tg = 1;
    EDX_REQUIRE(cfg.kw == 1 || cfg.kw == 2 || cfg.kw == 4 || cfg.kw == 6 || cfg.kw == 8 || cfg.kw == 12 ||
                    cfg.kw == 16 || cfg.kw == 32,
                "edx_krylov: apply_col_group must be one of 1, 2, 4, 6, 8, 12, 16, 32");
    EDX_REQUIRE(cfg.tg == 1 || cfg.tg == 2 || cfg.tg == 4, "edx_krylov: apply_tiles must be 1, 2 or 4");
    EDX_REQUIRE(cfg.threads == 256 || cfg.threads == 1024, "edx_krylov: apply_threads must be 256 or 1024");
    EDX_REQUIRE(bps >= 1 && bps * cfg.threads <= 8 * 256, "edx_krylov: apply_blocks_per_sm out of range");
    cfg.gx = num_sms() * bps;
    const edx_packed* packed = opts ? opts->apply_packed : nullptr;
    if (packed) {
        EDX_REQUIRE(packed->nrows == n && packed->row_ptr && packed->diag &&
                        (packed->nnz == 0 || (packed->ent && packed->vals)) && packed->nval >= 0 &&
                        packed->nval <= EDX_PACK_VALUES_MAX && packed->vbits >= 0 && packed->vbits <= 31 &&
                        (packed->vbits > 0 || packed->nnz == 0 || packed->vidx),
                    "edx_krylov: apply_packed does not describe this matrix");
    }
    if (cfg.rowslot)
        EDX_REQUIRE(cfg.kw <= 16 && k <= cfg.kw, "edx_krylov: apply_rowslot needs k <= apply_col_group <= 16");
    const edx_kron* kron = opts ? opts->apply_kron : nullptr;
    int kron_cw = 0;
    if (kron) {
        if ((rc = kron_check(kron))) return rc;
        EDX_REQUIRE(kron->nrows == n, "edx_krylov: apply_kron describes %lld rows, the matrix has %lld",
                    (long long)kron->nrows, (long long)n);
        EDX_REQUIRE(!packed, "edx_krylov: give apply_packed or apply_kron, not both");
        kron_cw = kron_col_group(k, opts->apply_col_group);
    }
    const int kw = pow2_kw(k);  // layout of the element-wise recurrence kernels
    const int gy = (k + kw - 1) / kw;
    int gx = num_sms() * 8;
    if (kron) gx = std::max(gx, kron_grid_x(kron, k, kron_cw, opts->apply_blocks_per_sm));
    Workspace w(d_work, work_bytes);
    KrylovWs ws;
    krylov_layout(w, n, k, nshift, maxn, gx, &ws);
    if (!ws.wbuf) return fail(EDX_ERR_WORKSPACE, "edx_krylov: workspace too small");

    KrylovState S;
    S.alpha_out = d_alpha;
    S.beta_out = d_beta;
    S.neff = d_neff;
    S.alpha = ws.alpha;
    S.beta = ws.beta;
    S.active = ws.active;
    S.n_active = ws.n_active;
    S.part = ws.part;
    S.ticket = ws.ticket;
    S.scur = ws.scur;
    S.sprev = ws.sprev;
    S.maxn = maxn;
    S.k = k;

    EDX_CUDA(cudaMemsetAsync(ws.ticket, 0, 4 * sizeof(unsigned), st));
    EDX_CUDA(cudaMemsetAsync(ws.kticket, 0, sizeof(unsigned) * (size_t)k, st));
    EDX_CUDA(cudaMemsetAsync(ws.kron_err, 0, sizeof(int), st));
    // tensor maps of the two Lanczos blocks for the slab product's staged loads (they swap
    // roles every step)
    alignas(64) CUtensorMap tm_c, tm_p;
    if (kron) {
        if ((rc = kron_tensor_map(kron, ws.Vc, k, kron_cw, &tm_c))) return rc;
        if ((rc = kron_tensor_map(kron, ws.Vp, k, kron_cw, &tm_p))) return rc;
    }
    EDX_CUDA(cudaMemsetAsync(ws.gticket, 0, sizeof(unsigned) * (size_t)((k + 31) / 32), st));
    EDX_CUDA(cudaMemsetAsync(d_alpha, 0, sizeof(double) * (size_t)k * maxn, st));
    EDX_CUDA(cudaMemsetAsync(d_beta, 0, sizeof(double) * (size_t)k * maxn, st));
    const double2* V0 = reinterpret_cast<const double2*>(d_v0);
    {
        dim3 grid(reduce_grid(n), gy);
        EDX_KW_SWITCH(kw, k_colnorm, grid, n, V0, ld0, S);
        EDX_CHECK_LAUNCH();
    }
    EDX_CUDA(cudaMemcpyAsync(d_norm, ws.alpha, sizeof(double) * k, cudaMemcpyDeviceToDevice, st));
    const int eb = (int)std::min<int64_t>((n * k + 255) / 256, (int64_t)num_sms() * 16);
    k_start<<<eb, 256, 0, st>>>(n, k, V0, ld0, ws.Vc, ws.Vp, ws.beta);
    EDX_CHECK_LAUNCH();
    if (nshift > 0) {
        EDX_CUDA(cudaMemsetAsync(ws.wbuf, 0, sizeof(double2) * 2 * (size_t)nshift * maxn, st));
        EDX_CUDA(cudaMemsetAsync(opts->shift_y, 0, sizeof(double2) * (size_t)nshift * maxn, st));
        k_shift_init<<<(nshift + 127) / 128, 128, 0, st>>>(nshift, opts->shift_col, ws.alpha, ws.sst,
                                                           opts->shift_tol, opts->shift_maxit);
        EDX_CHECK_LAUNCH();
    }
    // streaming projections: slots [0, win_n) of the window hold v_{win_i0 ..}
    int win_i0 = 0, win_n = 0;
    auto flush = [&]() -> int {
        if (!win || win_n == 0) return EDX_OK;
        for (int p = 0; p < nproj; ++p) {
            const int64_t m = opts->proj[p].nrows;
            const int64_t tot = m * (int64_t)opts->nacc;
            const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)num_sms() * 16);
            k_proj_accum<<<blocks, 256, 0, st>>>(m, win, win_n, win_i0, maxn, opts->nacc, opts->acc_col,
                                                 reinterpret_cast<const double2*>(opts->acc_coef),
                                                 reinterpret_cast<const double2*>(opts->proj_out[p]),
                                                 reinterpret_cast<double2*>(opts->acc_out[p]), opts->acc_ld);
            EDX_CHECK_LAUNCH();
        }
        win_i0 += win_n;
        win_n = 0;
        return EDX_OK;
    };
    auto project = [&](const double2* V, int i) -> int {
        const int slot = win ? i - win_i0 : i;
        const int64_t depth = win ? win : maxn;
        for (int p = 0; p < nproj; ++p) {
            const edx_csr* P = &opts->proj[p];
            double2* out = reinterpret_cast<double2*>(opts->proj_out[p]) + (int64_t)slot * P->nrows;
            int r2 = spmm_dispatch(P, k, EDX_C128, V, k, out, 1, depth * P->nrows,
                                   make_double2(1, 0), make_double2(0, 0), make_double2(0, 0), 0, st);
            if (r2) return r2;
            if (i > 0) {  // the stored vectors are unnormalised: scale to v_i
                const int64_t tot = P->nrows * (int64_t)k;
                const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)num_sms() * 8);
                k_proj_scale<<<blocks, 256, 0, st>>>(P->nrows, k, depth, slot,
                                                     reinterpret_cast<double2*>(opts->proj_out[p]), ws.scur);
                EDX_CHECK_LAUNCH();
            }
        }
        if (win && ++win_n == win) return flush();
        return EDX_OK;
    };
    if ((rc = project(ws.Vc, 0))) return rc;

    double2* Vc = ws.Vc;
    double2* Vp = ws.Vp;
    const int poll = 8;
    const bool timed = opts && opts->apply_ms;
    std::vector<cudaEvent_t> evs;
    auto drop_events = [&]() {
        for (auto e : evs) cudaEventDestroy(e);
        evs.clear();
    };
    int launches = 0;
    for (int it = 0; it < maxn; ++it) {
        // active-column count (summed by the orthogonalisation) and open-shift count
        EDX_CUDA(cudaMemsetAsync(ws.n_active, 0, (nshift > 0 ? 2 : 1) * sizeof(int), st));
        if (timed) {
            cudaEvent_t e0, e1;
            EDX_CUDA(cudaEventCreate(&e0));
            EDX_CUDA(cudaEventCreate(&e1));
            evs.push_back(e0);
            evs.push_back(e1);
            EDX_CUDA(cudaEventRecord(e0, st));
        }
        if (kron)
            rc = apply_kron(kron, Vc == ws.Vc ? static_cast<const void*>(&tm_c) : static_cast<const void*>(&tm_p), Vc,
                            Vp, S, it, ws.kticket, ws.kron_err, kron_cw, opts->apply_blocks_per_sm, st);
        else if (packed)
            rc = apply_packed(packed, Vc, Vp, S, it, cfg, st);
        else
            rc = (A->val_type == EDX_C128) ? apply_v<double2>(A, Vc, Vp, S, it, cfg, st)
                                           : apply_v<float2>(A, Vc, Vp, S, it, cfg, st);
        if (rc) {
            drop_events();
            return rc;
        }
        if (timed) EDX_CUDA(cudaEventRecord(evs.back(), st));
        ++launches;
        {
            dim3 grid(reduce_grid(n), gy);
            EDX_KW_SWITCH(kw, k_lanczos_orth, grid, n, Vc, Vp, S, ws.gticket, it);
            EDX_CHECK_LAUNCH();
        }
        if (nshift > 0) {
            k_shift_step<<<(nshift * 32 + 255) / 256, 256, 0, st>>>(
                nshift, opts->shift_col, reinterpret_cast<const double2*>(opts->shift_z), ws.sst, ws.wbuf,
                reinterpret_cast<double2*>(opts->shift_y), S, it, opts->shift_tol, opts->shift_maxit, ws.n_open);
            EDX_CHECK_LAUNCH();
        }
        std::swap(Vc, Vp);
        if (it + 1 < maxn && (rc = project(Vc, it + 1))) return rc;
        if ((it + 1) % poll == 0 || it + 1 == maxn) {
            int h[3] = {0, 0, 0};
            EDX_CUDA(cudaMemcpyAsync(h, ws.n_active, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
            EDX_CUDA(cudaStreamSynchronize(st));
            if (h[2]) {
                drop_events();
                if (h[2] == 2) return fail(EDX_ERR_INVALID, "edx_krylov: the slab form is inconsistent (a slab or a source row out of range)");
                return fail(EDX_ERR_CUDA, "edx_krylov: a staged slab load did not arrive within its time limit");
            }
            if (h[0] == 0) break;
            if (nshift > 0 && h[1] == 0) break;
        }
    }
    if ((rc = flush())) {
        drop_events();
        return rc;
    }
    if (nshift > 0) {
        k_shift_final<<<(nshift + 127) / 128, 128, 0, st>>>(nshift, ws.sst, opts->shift_iters, opts->shift_res);
        EDX_CHECK_LAUNCH();
    }
    if (timed) {
        EDX_CUDA(cudaStreamSynchronize(st));
        double total = 0.0;
        for (size_t q = 0; q + 1 < evs.size(); q += 2) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, evs[q], evs[q + 1]) == cudaSuccess) total += ms;
        }
        drop_events();
        *opts->apply_ms = total;
        if (opts->apply_launches) *opts->apply_launches = launches;
    } else if (opts && opts->apply_launches) {
        *opts->apply_launches = launches;
    }
    return EDX_OK;
}
