// edx_kron.cu -- the slab (impurity x bath) product: k_lanczos_apply_kron (fused Lanczos step
// and plain Y = H X), edx_kron_spmm, edx_permute_rows.
//
// In the slab order every row of slab s (impurity/core configuration I, m bath electrons)
// takes its inputs from a short list of whole source slabs (edx_kron.src_*): the slabs of
// H_A's row s, and the slabs I + a / I - a one bath electron away.  A block owns a run of
// slabs for CW columns; one thread stages each source slab into a ring of shared-memory
// buffers with 2-D tiled tensor loads (cp.async.bulk.tensor, 32-row boxes, completion on an
// mbarrier; no multicast), and every thread accumulates its rows x one column from shared
// memory: a scaled copy for H_A sources, and for hybridisation sources one bath-electron hop
// per occupied (or empty) bath orbital, whose target row is a table lookup.  So the only
// global traffic is the source slabs (from L2, contiguous rows), the block's own output rows
// and a few KB of tables; no matrix entries are streamed.
//
// Every wait on a staged load is bounded (KR_WAIT_LIMIT rounds of mbarrier.try_wait): a load
// that never arrives sets the error flag, the block waits (again bounded) for the loads it
// still has in flight and returns, and the host reports EDX_ERR_CUDA.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "edx_krylov.cuh"
#include "edx_spmm.cuh"

namespace edx {

constexpr int KR_NT = 256;       // threads per block
constexpr int KR_CW = 8;         // columns per column tile: one 128-byte line per staged row
constexpr int KR_BOXR = 32;      // rows per tensor-load box
constexpr int KR_NBUF = 3;       // source slabs staged ahead
constexpr uint32_t KR_WAIT_LIMIT = 1u << 21;

struct KronView {
    const int32_t* slab_off;
    const int32_t* slab_m;
    const uint32_t* slab_cfg;
    const int32_t* hyb_a;
    const double2* t_cre;
    const double2* t_ann;
    const int64_t* src_ptr;
    const int32_t* src_slab;
    const int32_t* src_kind;
    const double2* src_coef;
    const int32_t* b_off;
    const uint16_t* b_cfg;
    const uint16_t* b_nbr;
    const double2* b_diag;
    int nslab, nb, nah, n_alo;
};

static KronView view_of(const edx_kron* K) {
    return KronView{K->slab_off,
                    K->slab_m,
                    K->slab_cfg,
                    K->hyb_a,
                    reinterpret_cast<const double2*>(K->t_cre),
                    reinterpret_cast<const double2*>(K->t_ann),
                    K->src_ptr,
                    K->src_slab,
                    K->src_kind,
                    reinterpret_cast<const double2*>(K->src_coef),
                    K->b_off,
                    K->b_cfg,
                    K->b_nbr,
                    reinterpret_cast<const double2*>(K->b_diag),
                    K->nslab,
                    K->nb,
                    K->nah,
                    K->n_alo};
}

// ---- mbarrier and tensor-load primitives (PTX ISA: mbarrier, cp.async.bulk.tensor) --------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// true once the phase with this parity has completed; false after KR_WAIT_LIMIT rounds
__device__ __noinline__ bool mbar_wait_bounded(uint64_t* b, unsigned parity) {
    for (uint32_t i = 0; i < KR_WAIT_LIMIT; ++i) {
        if (mbar_try_wait(b, parity)) return true;
        if (i >= 8) __nanosleep(128);
    }
    return false;
}
// 2-D tiled tensor load of one box into shared memory; completion counted on `bar`.  The
// innermost coordinate x is a multiple of 2 doubles (16 bytes) by construction.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// parity of the A-side sign (src/fock.f90:38-68) of c+_a c_b (cre) and c+_b c_a (ann) on a
// row of a slab with compressed A configuration cfg and m bath electrons; a = compressed
// index of the A orbital, n_alo = A orbitals below the bath (edrixs_b200/kron.py)
__device__ __forceinline__ int sig_cre(uint32_t cfg, int m, int a, int n_alo) {
    const uint32_t lo = (1u << n_alo) - 1u;
    return (__popc(cfg & lo) + __popc(cfg & ((1u << a) - 1u)) + (a >= n_alo ? m - 1 : 0)) & 1;
}
__device__ __forceinline__ int sig_ann(uint32_t cfg, int m, int a, int n_alo) {
    const uint32_t lo = (1u << n_alo) - 1u;
    return (__popc(cfg & ((1u << a) - 1u)) + (a >= n_alo ? m : 0) + __popc(cfg & lo) - (a < n_alo ? 1 : 0)) & 1;
}

// ---- the slab product ---------------------------------------------------------------------
// grid (gx, column tiles of KR_CW); block b owns slabs b, b + gx, ...; thread t owns rows
// t, t + KR_NT, ... (RPT of them) of each slab and all KC columns of the tile, so the
// per-hop work (neighbour rank, sign, coefficient) is paid once for KC columns.  A staged
// slab is rows of 8 complex values (128 bytes) laid out by the tensor unit's 128-byte
// swizzle: value (r, c) sits at r * 8 + (c ^ (r & 7)), so lanes reading different rows spread
// over the banks.  LANCZOS: the fused step of k_lanczos_apply_packed (W = scur (H U_i) -
// beta_{i-1} sprev U_{i-1} into Y = V_prev, alpha partials, the last block of each column
// tile finishes alpha in block order); otherwise Y = H X.
template <int KC, int RPT, bool LANCZOS>
__global__ void __launch_bounds__(KR_NT) k_lanczos_apply_kron(KronView K, const __grid_constant__ CUtensorMap tm,
                                                              const double2* __restrict__ X, double2* __restrict__ Y,
                                                              KrylovState S, int k, int it, int stage_rows,
                                                              unsigned* __restrict__ tile_ticket,
                                                              int* __restrict__ err) {
    constexpr int NW = KR_NT / 32;
    extern __shared__ __align__(1024) unsigned char kr_smem[];
    // swizzled tensor-load destinations start on a 1024-byte boundary: align explicitly (the
    // host asks for 1024 spare bytes)
    double2* stages = reinterpret_cast<double2*>(kr_smem + ((1024u - (smem_addr(kr_smem) & 1023u)) & 1023u));
    const int stage_elems = stage_rows * KR_CW;
    double2* tcre = stages + KR_NBUF * stage_elems;
    double2* tann = tcre + K.nah * K.nb;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tann + K.nah * K.nb);
    __shared__ double wred[NW][KC];
    __shared__ bool sh_last;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c0 = blockIdx.y * KR_CW;
    const int kc = min(KC, k - c0);  // columns of this tile that exist

    for (int i = tid; i < K.nah * K.nb; i += KR_NT) {
        tcre[i] = K.t_cre[i];
        tann[i] = K.t_ann[i];
    }
    if (tid == 0) {
        for (int b = 0; b < KR_NBUF; ++b) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // producer cursor (thread 0): the next source to stage is source p_beg + p_j of slab
    // p_slab (every slab has at least its own slab as a source)
    int p_slab = blockIdx.x, p_j = 0;
    int64_t p_beg = 0, p_end = 0;
    if (p_slab < K.nslab) {
        p_beg = K.src_ptr[p_slab];
        p_end = K.src_ptr[p_slab + 1];
    }
    unsigned issued = 0;
    auto issue_next = [&]() -> bool {
        while (p_slab < K.nslab && p_beg + p_j >= p_end) {
            p_slab += gridDim.x;
            p_j = 0;
            if (p_slab < K.nslab) {
                p_beg = K.src_ptr[p_slab];
                p_end = K.src_ptr[p_slab + 1];
            }
        }
        if (p_slab >= K.nslab) return false;
        const int sl = K.src_slab[p_beg + p_j];
        ++p_j;
        const int r0 = K.slab_off[sl];
        const int rows = K.slab_off[sl + 1] - r0;
        int nbox = (rows + KR_BOXR - 1) / KR_BOXR;
        if (nbox * KR_BOXR > stage_rows) {  // a slab longer than max_rows: stage what fits, report it
            atomicExch(err, 2);
            nbox = stage_rows / KR_BOXR;
        }
        const int st = (int)(issued % KR_NBUF);
        double2* dst = stages + st * stage_elems;
        mbar_expect_tx(&bar[st], (unsigned)(nbox * KR_BOXR * KR_CW * (int)sizeof(double2)));
        for (int bx = 0; bx < nbox; ++bx)
            tma_load_2d(dst + bx * KR_BOXR * KR_CW, &tm, 2 * c0, r0 + bx * KR_BOXR, &bar[st]);
        ++issued;
        return true;
    };
    if (tid == 0)
        for (int i = 0; i < KR_NBUF; ++i)
            if (!issue_next()) break;

    double bprev[KC], scur[KC], apart[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        bprev[j] = scur[j] = apart[j] = 0.0;
        if (LANCZOS && j < kc) {
            bprev[j] = it > 0 ? S.beta[c0 + j] * S.sprev[c0 + j] : 0.0;
            scur[j] = S.scur[c0 + j];
        }
    }
    const uint32_t full = (1u << K.nb) - 1u;
    unsigned consumed = 0;
    bool bad = false;
    for (int s = blockIdx.x; s < K.nslab && !bad; s += gridDim.x) {
        const int off = K.slab_off[s];
        const int Rs = K.slab_off[s + 1] - off;
        // rows this block stages and holds; a slab longer than max_rows is reported, not read past
        const int R = min(Rs, min(stage_rows, RPT * KR_NT));
        if (tid == 0 && R != Rs) atomicExch(err, 2);
        const int m = K.slab_m[s];
        const uint32_t cfg = K.slab_cfg[s];
        const int bo = K.b_off[m];
        const int64_t sb = K.src_ptr[s], se = K.src_ptr[s + 1];
        double2 acc[RPT][KC];
        uint32_t Bv[RPT];
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            const int r = tid + q * KR_NT;
            Bv[q] = r < R ? __ldg(K.b_cfg + bo + r) : 0u;
#pragma unroll
            for (int j = 0; j < KC; ++j) acc[q][j] = make_double2(0.0, 0.0);
        }
        for (int64_t js = sb; js < se; ++js) {
            const int st = (int)(consumed % KR_NBUF);
            const unsigned par = (consumed / KR_NBUF) & 1u;
            const bool ok = mbar_wait_bounded(&bar[st], par);
            if (ok) {
                const double2* Xs = stages + st * stage_elems;
                const int kind = K.src_kind[js];
                const int type = kind & 15, q = kind >> 4;
                if (type <= EDX_KRON_SRC_OWN) {
                    const double2 v0 = K.src_coef[js];
#pragma unroll
                    for (int qq = 0; qq < RPT; ++qq) {
                        const int r = tid + qq * KR_NT;
                        if (r < R) {
                            double2 v = v0;
                            if (type == EDX_KRON_SRC_OWN) {
                                const double2 d = __ldg(K.b_diag + bo + r);
                                v.x += d.x;
                                v.y += d.y;
                            }
                            const double2* xr = Xs + r * KR_CW;
#pragma unroll
                            for (int j = 0; j < KC; ++j) acc[qq][j] = fma_c(v, xr[j ^ (r & 7)], acc[qq][j]);
                        }
                    }
                } else {
                    const bool cre = type == EDX_KRON_SRC_CRE;
                    const int a = K.hyb_a[q];
                    const int sa = cre ? sig_cre(cfg, m, a, K.n_alo) : sig_ann(cfg, m, a, K.n_alo);
                    const double2* T = (cre ? tcre : tann) + q * K.nb;
#pragma unroll
                    for (int qq = 0; qq < RPT; ++qq) {
                        const int r = tid + qq * KR_NT;
                        if (r < R) {
                            const uint32_t B = Bv[qq];
                            const uint16_t* nbr = K.b_nbr + (size_t)(bo + r) * K.nb;
                            uint32_t bits = cre ? B : (~B & full);
                            while (bits) {
                                const int b = __ffs(bits) - 1;
                                bits &= bits - 1u;
                                const int rs = min((int)__ldg(nbr + b), stage_rows - 1);  // stays in the stage
                                double2 t = T[b];
                                if ((sa ^ __popc(B & ((1u << b) - 1u))) & 1) {
                                    t.x = -t.x;
                                    t.y = -t.y;
                                }
                                const double2* xr = Xs + rs * KR_CW;
#pragma unroll
                                for (int j = 0; j < KC; ++j) acc[qq][j] = fma_c(t, xr[j ^ (rs & 7)], acc[qq][j]);
                            }
                        }
                    }
                }
            }
            ++consumed;
            // every thread is done with this stage (and all agree whether a load was lost)
            bad = __syncthreads_or(!ok) != 0;
            if (bad) break;
            if (tid == 0) {
                fence_proxy_async();
                issue_next();
            }
        }
        if (bad) break;
#pragma unroll
        for (int qq = 0; qq < RPT; ++qq) {
            const int r = tid + qq * KR_NT;
            if (r < R) {
                const int64_t o = (int64_t)(off + r) * k + c0;
#pragma unroll
                for (int j = 0; j < KC; ++j) {
                    if (j < kc) {
                        if (LANCZOS) {
                            const double2 vc = X[o + j];
                            const double2 vp = Y[o + j];
                            double2 w = make_double2(-bprev[j] * vp.x, -bprev[j] * vp.y);
                            w.x = w.x + scur[j] * acc[qq][j].x;
                            w.y = w.y + scur[j] * acc[qq][j].y;
                            Y[o + j] = w;
                            apart[j] += vc.x * w.x + vc.y * w.y;  // Re(conj(U_i) w); alpha = scur * sum
                        } else {
                            Y[o + j] = acc[qq][j];
                        }
                    }
                }
            }
        }
    }
    if (bad) {
        if (tid == 0) {
            atomicExch(err, 1);
            // the loads still in flight land before the block's shared memory is released
            for (unsigned u = consumed - 1; u < issued; ++u) mbar_wait_bounded(&bar[u % KR_NBUF], (u / KR_NBUF) & 1u);
        }
        return;
    }
    if constexpr (LANCZOS) {
        // alpha partials: a fixed butterfly inside each warp, then the warps in order
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            double v = apart[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) wred[warp][j] = v;
        }
        __syncthreads();
        if (tid < kc) {
            double t = 0.0;
            for (int w = 0; w < NW; ++w) t += wred[w][tid];
            S.part[(int64_t)blockIdx.x * k + c0 + tid] = t;
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) sh_last = atomicAdd(&tile_ticket[blockIdx.y], 1u) == gridDim.x - 1u;
        __syncthreads();
        if (!sh_last) return;
        __threadfence();
        __shared__ double red[KR_NT];
        for (int j = 0; j < kc; ++j) {
            const int col = c0 + j;
            double t = 0.0;
            for (int b = tid; b < (int)gridDim.x; b += KR_NT) t += __ldcg(S.part + (int64_t)b * k + col);
            red[tid] = t;
            __syncthreads();
            for (int h = KR_NT / 2; h > 0; h >>= 1) {
                if (tid < h) red[tid] += red[tid + h];
                __syncthreads();
            }
            if (tid == 0) {
                const double a = S.scur[col] * red[0];
                S.alpha[col] = a;
                if (S.active[col]) S.alpha_out[(int64_t)col * S.maxn + it] = a;
            }
            __syncthreads();
        }
        if (tid == 0) tile_ticket[blockIdx.y] = 0u;
    }
}

// ---- the slab product for large slabs: source rows read from global memory ---------------
// When the largest slab does not fit the staged ring (more than about 590 rows of 128 bytes,
// which is 12 or more bath orbitals), or on request, every thread owns one slab-order row
// and the KC columns of its tile, finds its slab by a binary search of slab_off, and reads
// its source rows where they lie: the row of the same rank for H_A and own-slab sources
// (consecutive threads read consecutive rows), and per occupied (or empty) bath orbital the
// row that the bath table names for hybridisation sources.  A slab is contiguous and a few MB
// at most, so these reads mostly hit L2.  Grid (gx, column tiles of KC); block b owns rows
// b * KR_NT + t, (b + gx) * KR_NT + t, ...  Epilogue and alpha partials as above.  A source
// row outside its slab (an inconsistent slab form) is skipped and reported (err = 2).
constexpr int KG_HOPS = 2;  // hops whose source rows load together

// KC complex values of one row tile: 32-byte loads (two complex values each) when the tile
// starts on a 32-byte boundary and is full (even k, even KC), else 16-byte loads
__device__ __forceinline__ void ld_c2(const double2* p, double2& a, double2& b) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p));
}
template <int KC>
__device__ __forceinline__ void ld_tile(const double2* p, int kc, bool pairs, double2* xs) {
    if (KC % 2 == 0 && pairs) {
#pragma unroll
        for (int h = 0; h < KC / 2; ++h) ld_c2(p + 2 * h, xs[2 * h], xs[2 * h + 1]);
    } else {
#pragma unroll
        for (int j = 0; j < KC; ++j) xs[j] = j < kc ? ldx(p + j) : make_double2(0.0, 0.0);
    }
}

template <int KC, bool LANCZOS>
__global__ void __launch_bounds__(KR_NT, 2) k_lanczos_apply_kron_gather(KronView K, int64_t nrows,
                                                                     const double2* __restrict__ X,
                                                                     double2* __restrict__ Y, KrylovState S, int k,
                                                                     int it, unsigned* __restrict__ tile_ticket,
                                                                     int* __restrict__ err) {
    constexpr int NW = KR_NT / 32;
    extern __shared__ double2 kg_tab[];  // t_cre, then t_ann (nah x nb each)
    __shared__ double wred[NW][KC];
    __shared__ bool sh_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c0 = blockIdx.y * KC;
    const int kc = min(KC, k - c0);
    double2* tcre = kg_tab;
    double2* tann = kg_tab + K.nah * K.nb;
    for (int i = tid; i < K.nah * K.nb; i += KR_NT) {
        tcre[i] = K.t_cre[i];
        tann[i] = K.t_ann[i];
    }
    __syncthreads();
    double bprev[KC], scur[KC], apart[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        bprev[j] = scur[j] = apart[j] = 0.0;
        if (LANCZOS && j < kc) {
            bprev[j] = it > 0 ? S.beta[c0 + j] * S.sprev[c0 + j] : 0.0;
            scur[j] = S.scur[c0 + j];
        }
    }
    const uint32_t full = (1u << K.nb) - 1u;
    const bool pairs = (k % 2 == 0) && kc == KC;  // every row tile of this block is 32-byte aligned
    bool bad = false;
    for (int64_t i = (int64_t)blockIdx.x * KR_NT + tid; i < nrows; i += (int64_t)gridDim.x * KR_NT) {
        int lo = 0, hi = K.nslab - 1;  // the last slab with slab_off <= i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(K.slab_off + mid) <= i) lo = mid;
            else hi = mid - 1;
        }
        const int s = lo;
        const int off = __ldg(K.slab_off + s);
        const int r = (int)(i - off);
        const int m = __ldg(K.slab_m + s);
        const uint32_t cfg = __ldg(K.slab_cfg + s);
        const int bo = __ldg(K.b_off + m);
        const uint32_t B = __ldg(K.b_cfg + bo + r);
        const uint16_t* nbr = K.b_nbr + (size_t)(bo + r) * K.nb;
        double2 acc[KC];
#pragma unroll
        for (int j = 0; j < KC; ++j) acc[j] = make_double2(0.0, 0.0);
        const int64_t se = __ldg(K.src_ptr + s + 1);
        for (int64_t js = __ldg(K.src_ptr + s); js < se; ++js) {
            const int sl = __ldg(K.src_slab + js);
            const int kind = __ldg(K.src_kind + js);
            const int type = kind & 15, q = kind >> 4;
            const int soff = __ldg(K.slab_off + sl);
            const int srows = __ldg(K.slab_off + sl + 1) - soff;
            if (type <= EDX_KRON_SRC_OWN) {
                if (r >= srows) {
                    bad = true;
                    continue;
                }
                double2 v = K.src_coef[js];
                if (type == EDX_KRON_SRC_OWN) {
                    const double2 d = __ldg(K.b_diag + bo + r);
                    v.x += d.x;
                    v.y += d.y;
                }
                double2 xs[KC];
                ld_tile<KC>(X + (int64_t)(soff + r) * k + c0, kc, pairs, xs);
#pragma unroll
                for (int j = 0; j < KC; ++j) acc[j] = fma_c(v, xs[j], acc[j]);
            } else {
                if (q >= K.nah) {
                    bad = true;
                    continue;
                }
                const bool cre = type == EDX_KRON_SRC_CRE;
                const int a = __ldg(K.hyb_a + q);
                const int sa = cre ? sig_cre(cfg, m, a, K.n_alo) : sig_ann(cfg, m, a, K.n_alo);
                const double2* T = (cre ? tcre : tann) + q * K.nb;
                uint32_t bits = cre ? B : (~B & full);
                while (bits) {
                    double2 t[KG_HOPS];
                    int64_t row[KG_HOPS];
                    bool ok[KG_HOPS];
#pragma unroll
                    for (int h = 0; h < KG_HOPS; ++h) {
                        ok[h] = bits != 0u;
                        const int b = ok[h] ? __ffs(bits) - 1 : 0;
                        if (ok[h]) bits &= bits - 1u;
                        const int rs = ok[h] ? (int)__ldg(nbr + b) : 0;
                        if (rs >= srows) {
                            bad = true;
                            ok[h] = false;
                        }
                        row[h] = (int64_t)(soff + rs) * k + c0;
                        t[h] = T[b];
                        if ((sa ^ __popc(B & ((1u << b) - 1u))) & 1) {
                            t[h].x = -t[h].x;
                            t[h].y = -t[h].y;
                        }
                    }
                    double2 xs[KG_HOPS][KC];
#pragma unroll
                    for (int h = 0; h < KG_HOPS; ++h) {
                        if (ok[h]) {
                            ld_tile<KC>(X + row[h], kc, pairs, xs[h]);
                        } else {
#pragma unroll
                            for (int j = 0; j < KC; ++j) xs[h][j] = make_double2(0.0, 0.0);
                        }
                    }
#pragma unroll
                    for (int h = 0; h < KG_HOPS; ++h)
#pragma unroll
                        for (int j = 0; j < KC; ++j) acc[j] = fma_c(t[h], xs[h][j], acc[j]);
                }
            }
        }
        const int64_t o = i * k + c0;
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            if (j < kc) {
                if (LANCZOS) {
                    const double2 vc = X[o + j];
                    const double2 vp = Y[o + j];
                    double2 w = make_double2(-bprev[j] * vp.x, -bprev[j] * vp.y);
                    w.x = w.x + scur[j] * acc[j].x;
                    w.y = w.y + scur[j] * acc[j].y;
                    Y[o + j] = w;
                    apart[j] += vc.x * w.x + vc.y * w.y;  // Re(conj(U_i) w); alpha = scur * sum
                } else {
                    Y[o + j] = acc[j];
                }
            }
        }
    }
    if (bad) atomicExch(err, 2);
    if constexpr (LANCZOS) {
        // alpha partials: a fixed butterfly inside each warp, then the warps in order
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            double v = apart[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) wred[warp][j] = v;
        }
        __syncthreads();
        if (tid < kc) {
            double t = 0.0;
            for (int w = 0; w < NW; ++w) t += wred[w][tid];
            S.part[(int64_t)blockIdx.x * k + c0 + tid] = t;
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) sh_last = atomicAdd(&tile_ticket[blockIdx.y], 1u) == gridDim.x - 1u;
        __syncthreads();
        if (!sh_last) return;
        __threadfence();
        __shared__ double red[KR_NT];
        for (int j = 0; j < kc; ++j) {
            const int col = c0 + j;
            double t = 0.0;
            for (int b = tid; b < (int)gridDim.x; b += KR_NT) t += __ldcg(S.part + (int64_t)b * k + col);
            red[tid] = t;
            __syncthreads();
            for (int h = KR_NT / 2; h > 0; h >>= 1) {
                if (tid < h) red[tid] += red[tid + h];
                __syncthreads();
            }
            if (tid == 0) {
                const double a = S.scur[col] * red[0];
                S.alpha[col] = a;
                if (S.active[col]) S.alpha_out[(int64_t)col * S.maxn + it] = a;
            }
            __syncthreads();
        }
        if (tid == 0) tile_ticket[blockIdx.y] = 0u;
    }
}

// ---- host side ----------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// columns computed per thread: the smallest supported count >= k within the 8-column tile
static int kc_of(int k) {
    for (int w : {1, 2, 4, 6, 8})
        if (w >= k) return w;
    return 8;
}

static int stage_rows_of(const edx_kron* K) { return (K->max_rows + KR_BOXR - 1) / KR_BOXR * KR_BOXR; }

static size_t smem_bytes(const edx_kron* K) {
    return 1024 + (size_t)KR_NBUF * stage_rows_of(K) * KR_CW * sizeof(double2) +
           2 * (size_t)K->nah * K->nb * sizeof(double2) + KR_NBUF * sizeof(uint64_t);
}

static int rpt_of(const edx_kron* K) {
    for (int r : {1, 2, 4})
        if (r * KR_NT >= K->max_rows) return r;
    return 0;
}

int kron_check(const edx_kron* K) {
    EDX_REQUIRE(K != nullptr, "slab form: NULL descriptor");
    EDX_REQUIRE(K->nrows >= 1 && K->nrows < ((int64_t)1 << 31) && K->nslab >= 1 && K->nb >= 1 &&
                    K->nb <= EDX_KRON_NB_MAX && K->nah >= 0 && K->nah <= EDX_KRON_NAH_MAX && K->n_alo >= 0 &&
                    K->n_alo <= 31 && K->max_rows >= 1,
                "slab form: sizes out of range (nrows %lld, nslab %d, nb %d, nah %d)", (long long)K->nrows,
                K->nslab, K->nb, K->nah);
    EDX_REQUIRE(K->slab_off && K->slab_m && K->slab_cfg && K->src_ptr && K->src_slab && K->src_kind && K->src_coef &&
                    K->b_off && K->b_cfg && K->b_nbr && K->b_diag && (K->nah == 0 || (K->hyb_a && K->t_cre && K->t_ann)),
                "slab form: a device array is missing");
    return EDX_OK;
}

// the staged product needs every slab within one block (4 rows per thread at most) and the
// ring of staged slabs within shared memory
static bool staged_fits(const edx_kron* K) { return rpt_of(K) != 0 && smem_bytes(K) + 8 * 1024 <= 227 * 1024; }
// AUTO: the gather product for up to 8 columns (one tile: 0.70 against 0.89 ms on a 1 M-row
// impurity H_n) and whenever the staged ring does not fit; the staged product for wider
// blocks (96 columns: 2.1 against 2.9 ms; 768: 16.5 against 22.3 ms)
static bool gather_of(const edx_kron* K, int variant, int k) {
    return variant == EDX_KRON_GATHER || !staged_fits(K) || (variant != EDX_KRON_STAGED && k <= KR_CW);
}
// columns per thread of the gather product: the smallest supported count >= k, 8 beyond
static int gather_kc(int k) { return kc_of(k); }

int kron_grid_x(const edx_kron* K, int k, int variant, int blocks_per_sm) {
    if (gather_of(K, variant, k)) {
        const int kc = gather_kc(k);
        const int ntile = (k + kc - 1) / kc;
        // blocks_per_sm x SMs blocks in all (0: 8 blocks of 256 threads per SM, 4 rounds)
        const int64_t target = (int64_t)num_sms() * (blocks_per_sm > 0 ? blocks_per_sm : 8 * 4);
        const int64_t gx = (target + ntile - 1) / ntile;
        const int64_t need = (K->nrows + KR_NT - 1) / KR_NT;
        return (int)std::max<int64_t>(1, std::min(gx, need));
    }
    const size_t sm = smem_bytes(K);
    int occ = (int)std::min<size_t>(8, (size_t)(227 * 1024) / std::max<size_t>(sm + 2048, 1));
    if (occ < 1) occ = 1;
    const int ntile = (k + KR_CW - 1) / KR_CW;
    const int64_t target = (int64_t)num_sms() * occ * 4;
    int64_t gx = (target + ntile - 1) / ntile;
    gx = std::max<int64_t>(1, std::min<int64_t>(gx, K->nslab));
    return (int)gx;
}

// 2-D tensor map of an n x k complex128 block (row-major) as doubles, boxes of 32 rows x 8
// complex values, 128-byte swizzle.  Columns past k (k < 8, or the last tile) read as zeros.
int kron_tensor_map(const edx_kron* K, const double2* X, int k, int /*col_group*/, void* out) {
    auto fn = encode_tiled();
    if (!fn) return fail(EDX_ERR_CUDA, "slab form: cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[2] = {(cuuint64_t)2 * k, (cuuint64_t)K->nrows};
    cuuint64_t strides[1] = {(cuuint64_t)2 * k * sizeof(double)};
    cuuint32_t box[2] = {(cuuint32_t)(2 * KR_CW), (cuuint32_t)KR_BOXR};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double2*>(X),
                    dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(EDX_ERR_CUDA, "slab form: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return EDX_OK;
}

template <int KC, int RPT, bool LANCZOS>
static int launch_kron_rpt(const edx_kron* K, const CUtensorMap* tm, const double2* X, double2* Y, const KrylovState& S,
                           int k, int it, unsigned* tt, int* err, cudaStream_t st) {
    auto kern = k_lanczos_apply_kron<KC, RPT, LANCZOS>;
    const size_t sm = smem_bytes(K);
    // the attribute is the most this kernel can be given (the device's opt-in limit less its
    // static shared memory), the same on every call: threads launching for different slab
    // forms at once must not lower it under one another's launch
    int dev = 0, optin = 0;
    EDX_CUDA(cudaGetDevice(&dev));
    EDX_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    EDX_CUDA(cudaFuncGetAttributes(&fa, kern));
    const size_t max_dyn = (size_t)optin - fa.sharedSizeBytes;
    EDX_REQUIRE(sm <= max_dyn, "slab form: %zu bytes of staged slabs exceed shared memory", sm);
    EDX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_dyn));
    const int ntile = (k + KR_CW - 1) / KR_CW;
    EDX_REQUIRE(ntile <= 65535, "slab form: too many column tiles");
    dim3 grid(kron_grid_x(K, k, 0, 0), ntile);
    kern<<<grid, KR_NT, sm, st>>>(view_of(K), *tm, X, Y, S, k, it, stage_rows_of(K), tt, err);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <int KC, bool LANCZOS>
static int launch_kron_kc(const edx_kron* K, const CUtensorMap* tm, const double2* X, double2* Y, const KrylovState& S,
                          int k, int it, unsigned* tt, int* err, cudaStream_t st) {
    switch (rpt_of(K)) {
    case 1: return launch_kron_rpt<KC, 1, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    case 2: return launch_kron_rpt<KC, 2, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    case 4: return launch_kron_rpt<KC, 4, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    }
    return fail(EDX_ERR_INVALID, "slab form: slabs of %d rows exceed the %d rows a block holds", K->max_rows,
                4 * KR_NT);
}

template <int KC, bool LANCZOS>
static int launch_gather_kc(const edx_kron* K, const double2* X, double2* Y, const KrylovState& S, int k, int it,
                            unsigned* tt, int* err, int bps, cudaStream_t st) {
    auto kern = k_lanczos_apply_kron_gather<KC, LANCZOS>;
    const size_t sm = 2 * (size_t)K->nah * K->nb * sizeof(double2);
    const int ntile = (k + KC - 1) / KC;
    EDX_REQUIRE(ntile <= 65535, "slab form: too many column tiles");
    dim3 grid(kron_grid_x(K, k, EDX_KRON_GATHER, bps), ntile);
    kern<<<grid, KR_NT, sm, st>>>(view_of(K), K->nrows, X, Y, S, k, it, tt, err);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

template <bool LANCZOS>
static int launch_kron(const edx_kron* K, const CUtensorMap* tm, const double2* X, double2* Y, const KrylovState& S,
                       int k, int it, unsigned* tt, int* err, int variant, int bps, cudaStream_t st) {
    if (variant == EDX_KRON_STAGED && !staged_fits(K))
        return fail(EDX_ERR_INVALID, "slab form: slabs of %d rows do not fit the staged product's shared memory",
                    K->max_rows);
    if (gather_of(K, variant, k)) {
        switch (gather_kc(k)) {
        case 1: return launch_gather_kc<1, LANCZOS>(K, X, Y, S, k, it, tt, err, bps, st);
        case 2: return launch_gather_kc<2, LANCZOS>(K, X, Y, S, k, it, tt, err, bps, st);
        case 4: return launch_gather_kc<4, LANCZOS>(K, X, Y, S, k, it, tt, err, bps, st);
        case 6: return launch_gather_kc<6, LANCZOS>(K, X, Y, S, k, it, tt, err, bps, st);
        default: return launch_gather_kc<8, LANCZOS>(K, X, Y, S, k, it, tt, err, bps, st);
        }
    }
    switch (kc_of(k)) {
    case 1: return launch_kron_kc<1, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    case 2: return launch_kron_kc<2, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    case 4: return launch_kron_kc<4, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    case 6: return launch_kron_kc<6, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    default: return launch_kron_kc<8, LANCZOS>(K, tm, X, Y, S, k, it, tt, err, st);
    }
}

// the product variant a caller's apply_col_group selects (EDX_KRON_AUTO / _STAGED / _GATHER;
// other values: automatic)
int kron_col_group(int /*k*/, int requested) {
    return (requested == EDX_KRON_STAGED || requested == EDX_KRON_GATHER) ? requested : EDX_KRON_AUTO;
}

int apply_kron(const edx_kron* K, const void* tmap, const double2* Vc, double2* Vp, const KrylovState& S, int it,
               unsigned* tile_ticket, int* err, int col_group, int blocks_per_sm, cudaStream_t st) {
    return launch_kron<true>(K, static_cast<const CUtensorMap*>(tmap), Vc, Vp, S, S.k, it, tile_ticket, err,
                             kron_col_group(S.k, col_group), blocks_per_sm, st);
}

__global__ void k_permute_rows(int64_t n, int k, const double2* __restrict__ src, int64_t lds,
                               const int64_t* __restrict__ idx, double2* __restrict__ dst, int64_t ldd) {
    const int64_t tot = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / k;
        const int c = (int)(e - i * k);
        dst[i * ldd + c] = __ldg(src + __ldg(idx + i) * lds + c);
    }
}

}  // namespace edx

using namespace edx;

extern "C" int edx_kron_spmm_workspace(size_t* bytes) {
    EDX_REQUIRE(bytes != nullptr, "edx_kron_spmm_workspace: bad arguments");
    *bytes = 256;
    return EDX_OK;
}

extern "C" int edx_kron_spmm(const edx_kron* K, int k, const double* d_x, double* d_y, int col_group, void* d_work,
                             size_t work_bytes, void* stream) {
    int rc = kron_check(K);
    if (rc) return rc;
    EDX_REQUIRE(k >= 1 && d_x && d_y && d_x != d_y, "edx_kron_spmm: bad arguments");
    const int variant = kron_col_group(k, col_group);
    Workspace w(d_work, work_bytes);
    int* err = w.take<int>(1);
    if (!err) return fail(EDX_ERR_WORKSPACE, "edx_kron_spmm: workspace too small");
    cudaStream_t st = as_stream(stream);
    EDX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    alignas(64) CUtensorMap tm;
    if (!gather_of(K, variant, k) && (rc = kron_tensor_map(K, reinterpret_cast<const double2*>(d_x), k, 0, &tm)))
        return rc;
    KrylovState S{};
    rc = launch_kron<false>(K, &tm, reinterpret_cast<const double2*>(d_x), reinterpret_cast<double2*>(d_y), S, k, 0,
                            nullptr, err, variant, 0, st);
    if (rc) return rc;
    int h = 0;
    EDX_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    if (h == 2) return fail(EDX_ERR_INVALID, "edx_kron_spmm: the slab form is inconsistent (a slab or a source row out of range)");
    if (h) return fail(EDX_ERR_CUDA, "edx_kron_spmm: a staged slab load did not arrive within its time limit");
    return EDX_OK;
}

extern "C" int edx_permute_rows(int64_t n, int k, const double* d_src, int64_t ld_src, const int64_t* d_idx,
                                double* d_dst, int64_t ld_dst, void* stream) {
    EDX_REQUIRE(n >= 0 && k >= 1 && ld_src >= k && ld_dst >= k && (n == 0 || (d_src && d_idx && d_dst)) &&
                    d_src != d_dst,
                "edx_permute_rows: bad arguments");
    if (n == 0) return EDX_OK;
    cudaStream_t st = as_stream(stream);
    const int blocks = (int)std::min<int64_t>((n * k + 255) / 256, (int64_t)num_sms() * 16);
    k_permute_rows<<<blocks, 256, 0, st>>>(n, k, reinterpret_cast<const double2*>(d_src), ld_src, d_idx,
                                           reinterpret_cast<double2*>(d_dst), ld_dst);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}
