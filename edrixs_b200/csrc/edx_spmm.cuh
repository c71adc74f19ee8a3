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

// Lane layout of a warp working on one row: lane = slot * KW + c with SLOTS = 32 / KW slots
// (KW need not be a power of two; lanes beyond SLOTS*KW idle).  The warp streams the row's
// nonzeros in chunks of 32 (one coalesced load per lane); each slot takes every SLOTS-th
// entry of a chunk by shuffle.  This product is bound by gather latency, so the loops below
// issue several independent gathers before consuming any of them.
template <int KW>
struct Slots {
    static constexpr int N = 32 / KW;
    static constexpr bool POW2 = (KW & (KW - 1)) == 0;
};

// Row r times TG column tiles of X (columns (tile0 + g)*KW + c, g < TG) with explicit
// memory-level parallelism: per chunk of 32 nonzeros, U entries per slot are shuffled out
// first, then all U*TG gathers are issued, then the FMAs run.  acc[g] holds the row sum of
// tile g in every lane of column c on return.  Lanes with slot >= SLOTS idle.
template <int KW, int TG, class VT, class XT>
__device__ __forceinline__ void row_times_x_tiles(int64_t start, int64_t end, const int32_t* __restrict__ col,
                                                  const VT* __restrict__ val, const XT* __restrict__ X,
                                                  int64_t ldx_, int col0, int k, typename Acc<VT, XT>::T* acc) {
    using AT = typename Acc<VT, XT>::T;
    constexpr int SLOTS = Slots<KW>::N;
    constexpr int GROUPS = (32 + SLOTS - 1) / SLOTS;          // entry groups per chunk
    constexpr int U0 = (8 / TG) > 0 ? (8 / TG) : 1;           // gathers in flight per lane ~ 8
    constexpr int U = U0 < GROUPS ? U0 : GROUPS;
    const int lane = threadIdx.x & 31;
    const int slot = lane / KW;
    const int c = lane % KW;
    const bool slot_ok = slot < SLOTS;
    bool colok[TG];
#pragma unroll
    for (int g = 0; g < TG; ++g) {
        colok[g] = slot_ok && (col0 + g * KW + c < k);
        acc[g] = zero_c<AT>();
    }
    if (KW == 1) {
        // each lane owns its own entries; U1 rounds of 32 per pass, so a typical row
        // issues all its loads at once
        constexpr int U1 = 4;
        for (int64_t base = start; base < end; base += 32 * U1) {
            int cc[U1];
            AT vv[U1];
#pragma unroll
            for (int u = 0; u < U1; ++u) {
                const int64_t j = base + u * 32 + lane;
                cc[u] = 0;
                vv[u] = zero_c<AT>();
                if (j < end) {
                    cc[u] = ld_stream(col + j);
                    vv[u] = to_acc(ld_stream(val + j), AT());
                }
            }
            AT xs[U1][TG];
#pragma unroll
            for (int u = 0; u < U1; ++u)
#pragma unroll
                for (int g = 0; g < TG; ++g) {
                    xs[u][g] = zero_c<AT>();
                    if (base + u * 32 + lane < end && colok[g])
                        xs[u][g] = to_acc(ldx(X + (int64_t)cc[u] * ldx_ + col0 + g), AT());
                }
#pragma unroll
            for (int u = 0; u < U1; ++u)
#pragma unroll
                for (int g = 0; g < TG; ++g) acc[g] = fma_c(vv[u], xs[u][g], acc[g]);
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
#pragma unroll
            for (int q0 = 0; q0 < GROUPS; q0 += U) {
                int cc[U];
                AT vv[U];
                bool ok[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int src = (q0 + u) * SLOTS + slot;
                    cc[u] = __shfl_sync(0xffffffffu, cj, src & 31);
                    VT t = shfl2(vj, src & 31);
                    vv[u] = to_acc(t, AT());
                    ok[u] = (q0 + u < GROUPS) && src < cnt;
                }
                AT xs[U][TG];
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int g = 0; g < TG; ++g) {
                        xs[u][g] = zero_c<AT>();
                        if (ok[u] && colok[g])
                            xs[u][g] = to_acc(ldx(X + (int64_t)cc[u] * ldx_ + col0 + g * KW + c), AT());
                    }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int g = 0; g < TG; ++g) acc[g] = fma_c(vv[u], xs[u][g], acc[g]);
            }
        }
    }
#pragma unroll
    for (int g = 0; g < TG; ++g) {
        if (Slots<KW>::POW2) {
#pragma unroll
            for (int off = KW; off < 32; off <<= 1) acc[g] = xor_sum(acc[g], off);
        } else {
            AT tot = zero_c<AT>();
#pragma unroll
            for (int s = 0; s < SLOTS; ++s) {
                AT o;
                o.x = __shfl_sync(0xffffffffu, acc[g].x, s * KW + c);
                o.y = __shfl_sync(0xffffffffu, acc[g].y, s * KW + c);
                tot = add_c(tot, o);
            }
            acc[g] = tot;
        }
    }
}

// One column, long rows: a warp walks rows r0, r0 + rstep, ...; each row's first 128 entries
// are held four per lane, and the next row's entries load while this row's x values are
// gathered, so a row pays one memory latency instead of two.  Rows longer than 128
// entries finish their tail with plain 32-entry rounds.  epi(r, sum) is called with the
// row's sum in every lane.  Per lane the sum runs over entries lane, lane + 32, ... in order,
// then the warp adds lanes by a butterfly, as row_times_x_tiles<1>.
template <class VT, class XT, class Epi>
__device__ __forceinline__ void spmv_rows(int64_t r0, int64_t r1, int64_t rstep, const int64_t* __restrict__ row_ptr,
                                          const int32_t* __restrict__ col, const VT* __restrict__ val,
                                          const XT* __restrict__ X, int64_t ldx_, int col0, Epi epi) {
    using AT = typename Acc<VT, XT>::T;
    const int lane = threadIdx.x & 31;
    if (r0 >= r1) return;
    int cc[4];
    AT vv[4];
    int64_t s = __ldg(row_ptr + r0), e = __ldg(row_ptr + r0 + 1);
    auto load4 = [&](int64_t st, int64_t en, int* c4, AT* v4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t j = st + u * 32 + lane;
            c4[u] = j < en ? ld_stream(col + j) : 0;
            v4[u] = j < en ? to_acc(ld_stream(val + j), AT()) : zero_c<AT>();
        }
    };
    load4(s, e, cc, vv);
    for (int64_t r = r0; r < r1; r += rstep) {
        const int64_t rn = r + rstep;
        int64_t sn = 0, en = 0;
        int cn[4];
        AT vn[4];
        if (rn < r1) {
            sn = __ldg(row_ptr + rn);
            en = __ldg(row_ptr + rn + 1);
        }
        load4(sn, en, cn, vn);  // next row's entries (none past the last row)
        AT acc = zero_c<AT>();
        AT xs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            xs[u] = (s + u * 32 + lane < e) ? to_acc(ldx(X + (int64_t)cc[u] * ldx_ + col0), AT()) : zero_c<AT>();
#pragma unroll
        for (int u = 0; u < 4; ++u) acc = fma_c(vv[u], xs[u], acc);
        for (int64_t base = s + 128; base < e; base += 32) {  // tail of a long row
            const int64_t j = base + lane;
            if (j < e)
                acc = fma_c(to_acc(ld_stream(val + j), AT()),
                            to_acc(ldx(X + (int64_t)ld_stream(col + j) * ldx_ + col0), AT()), acc);
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) acc = xor_sum(acc, off);
        epi(r, acc);
        s = sn;
        e = en;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            cc[u] = cn[u];
            vv[u] = vn[u];
        }
    }
}

// The same for rows of up to ~100 entries: each half-warp owns a row (two rows per warp in
// flight), holds its first 16 * NC entries NC per lane and loads the next row's while this
// one's x values are gathered, so fewer lanes idle at the end of a row than with 32 lanes on
// a 60-100 entry row.  NC = 5 for rows of up to ~75 entries on average, else 6.  Half h of the warp takes rows 2p + h for pairs p = p0, p0 + pstep, ...
// below ceil(nrows / 2); epi(r, sum) is called with the row's sum in every lane of the half.
template <int NC, class VT, class XT, class Epi>
__device__ __forceinline__ void spmv_rows_half(int64_t p0, int64_t pstep, int64_t nrows,
                                               const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                                               const VT* __restrict__ val, const XT* __restrict__ X, int64_t ldx_,
                                               int col0, Epi epi) {
    using AT = typename Acc<VT, XT>::T;
    const int lane = threadIdx.x & 31;
    const int h = lane >> 4, l = lane & 15;
    const int64_t np = (nrows + 1) / 2;
    if (p0 >= np) return;
    int cc[NC];
    AT vv[NC];
    auto bounds = [&](int64_t p, int64_t& st, int64_t& en) {
        const int64_t r = 2 * p + h;
        st = en = 0;
        if (p < np && r < nrows) {
            st = __ldg(row_ptr + r);
            en = __ldg(row_ptr + r + 1);
        }
    };
    auto loadc = [&](int64_t st, int64_t en, int* c, AT* v) {
#pragma unroll
        for (int u = 0; u < NC; ++u) {
            const int64_t j = st + u * 16 + l;
            c[u] = j < en ? ld_stream(col + j) : 0;
            v[u] = j < en ? to_acc(ld_stream(val + j), AT()) : zero_c<AT>();
        }
    };
    int64_t s, e;
    bounds(p0, s, e);
    loadc(s, e, cc, vv);
    for (int64_t p = p0; p < np; p += pstep) {
        int64_t sn, en;
        bounds(p + pstep, sn, en);
        int cn[NC];
        AT vn[NC];
        loadc(sn, en, cn, vn);  // next row's entries (none past the last row)
        AT acc = zero_c<AT>();
        AT xs[NC];
#pragma unroll
        for (int u = 0; u < NC; ++u)
            xs[u] = (s + u * 16 + l < e) ? to_acc(ldx(X + (int64_t)cc[u] * ldx_ + col0), AT()) : zero_c<AT>();
#pragma unroll
        for (int u = 0; u < NC; ++u) acc = fma_c(vv[u], xs[u], acc);
        for (int64_t base = s + NC * 16; base < e; base += 16) {  // tail of a long row
            const int64_t j = base + l;
            if (j < e)
                acc = fma_c(to_acc(ld_stream(val + j), AT()),
                            to_acc(ldx(X + (int64_t)ld_stream(col + j) * ldx_ + col0), AT()), acc);
        }
#pragma unroll
        for (int off = 1; off < 16; off <<= 1) acc = xor_sum(acc, off);
        const int64_t r = 2 * p + h;
        if (r < nrows) epi(r, acc);
        s = sn;
        e = en;
#pragma unroll
        for (int u = 0; u < NC; ++u) {
            cc[u] = cn[u];
            vv[u] = vn[u];
        }
    }
}

// Short rows (a transition operator has ~10 entries per row): each slot of the warp owns a
// row of its own and walks its entries, U at a time, with the slot's KW lanes reading the
// same entry (a broadcast) and gathering their own columns of X.  No cross-slot reduction.
template <int KW, class VT, class XT>
__device__ __forceinline__ void row_times_x_slot(int64_t start, int64_t end, const int32_t* __restrict__ col,
                                                 const VT* __restrict__ val, const XT* __restrict__ X,
                                                 int64_t ldx_, int gc, bool colok, typename Acc<VT, XT>::T& acc) {
    using AT = typename Acc<VT, XT>::T;
    constexpr int U = 4;
    acc = zero_c<AT>();
    for (int64_t base = start; base < end; base += U) {
        int cc[U];
        AT vv[U], xs[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool ok = base + u < end;
            cc[u] = ok ? __ldg(col + base + u) : 0;
            vv[u] = ok ? to_acc(__ldg(val + base + u), AT()) : zero_c<AT>();
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            xs[u] = (base + u < end && colok) ? to_acc(ldx(X + (int64_t)cc[u] * ldx_ + gc), AT()) : zero_c<AT>();
#pragma unroll
        for (int u = 0; u < U; ++u) acc = fma_c(vv[u], xs[u], acc);
    }
}

// Streaming loads of packed entry words (read once per product).
__device__ __forceinline__ uint4 ld_stream4(const uint32_t* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}
__device__ __forceinline__ uint32_t ld_stream1(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
                 : "=r"(v)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}

// device view of an edx_packed matrix
struct PackedView {
    const int64_t* row_ptr;
    const uint32_t* ent;
    const double2* vals;
    const double2* diag;
    int vbits, nval;
    const uint16_t* vidx;  // wide form (vbits == 0)
};

// 16-bit value indices of the wide packed form, streamed like the entry words
__device__ __forceinline__ uint32_t ld_stream_u16(const uint16_t* p) {
    unsigned short v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;"
                 : "=h"(v)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}
__device__ __forceinline__ uint2 ld_stream_u16x4(const uint16_t* p) {  // 4 indices, 8-byte aligned
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y)
                 : "l"(p), "l"(evict_first_policy()));
    return v;
}

// column and value index of one packed entry: narrow form w = column << vbits | index;
// wide form (WIDE) w = column, vi = index
template <bool WIDE>
__device__ __forceinline__ void pk_decode(uint32_t w, uint32_t vi, int vbits, uint32_t vmask, int64_t& col,
                                          uint32_t& idx) {
    if (WIDE) {
        col = (int64_t)w;
        idx = vi;
    } else {
        col = (int64_t)(w >> vbits);
        idx = w & vmask;
    }
}

// One-column product on the packed form, warp per row, as spmv_rows: lanes take entries
// lane, lane + 32, ... (coalesced word loads), the next row's first 128 words load while this
// row's gathers run, the value comes from the shared-memory table `tab`.
template <bool WIDE, class Epi>
__device__ __forceinline__ void spmv_rows_packed(int64_t r0, int64_t r1, int64_t rstep, const PackedView& M,
                                                 const double2* tab, const double2* __restrict__ X, int64_t ldx_,
                                                 int col0, Epi epi) {
    const int lane = threadIdx.x & 31;
    if (r0 >= r1) return;
    const uint32_t vmask = WIDE ? 0u : (1u << M.vbits) - 1u;
    uint32_t ww[4], wi[4];
    int64_t s = __ldg(M.row_ptr + r0), e = __ldg(M.row_ptr + r0 + 1);
    auto load4 = [&](int64_t st, int64_t en, uint32_t* w4, uint32_t* i4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t j = st + u * 32 + lane;
            w4[u] = j < en ? ld_stream1(M.ent + j) : 0u;
            i4[u] = (WIDE && j < en) ? ld_stream_u16(M.vidx + j) : 0u;
        }
    };
    load4(s, e, ww, wi);
    for (int64_t r = r0; r < r1; r += rstep) {
        const int64_t rn = r + rstep;
        int64_t sn = 0, en = 0;
        uint32_t wn[4], in_[4];
        if (rn < r1) {
            sn = __ldg(M.row_ptr + rn);
            en = __ldg(M.row_ptr + rn + 1);
        }
        load4(sn, en, wn, in_);
        double2 acc = make_double2(0.0, 0.0);
        double2 xs[4], vs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            int64_t cc;
            uint32_t q;
            pk_decode<WIDE>(ww[u], wi[u], M.vbits, vmask, cc, q);
            const bool ok = s + u * 32 + lane < e;
            xs[u] = ok ? ldx(X + cc * ldx_ + col0) : make_double2(0.0, 0.0);
            vs[u] = ok ? tab[q] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) acc = fma_c(vs[u], xs[u], acc);
        for (int64_t base = s + 128; base < e; base += 32) {  // tail of a long row
            const int64_t j = base + lane;
            if (j < e) {
                int64_t cc;
                uint32_t q;
                pk_decode<WIDE>(ld_stream1(M.ent + j), WIDE ? ld_stream_u16(M.vidx + j) : 0u, M.vbits, vmask, cc, q);
                acc = fma_c(tab[q], ldx(X + cc * ldx_ + col0), acc);
            }
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) acc = xor_sum(acc, off);
        epi(r, acc);
        s = sn;
        e = en;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            ww[u] = wn[u];
            wi[u] = in_[u];
        }
    }
}

// Off-diagonal part of row r of a packed matrix (values in the shared-memory table `tab`)
// times TG column tiles of X.  Same lane layout and result as row_times_x_tiles.  With one
// slot per warp (KW = 32) every lane walks the same entries, four words per 16-byte broadcast
// load (and four wide-form indices per 8-byte load), so an entry costs one table read and no
// shuffles.  With several slots, slot s takes entries start + s, start + s + SLOTS, ...; one
// load instruction fetches adjacent words for all slots.
template <int KW, int TG, bool WIDE>
__device__ __forceinline__ void row_times_x_packed(int64_t start, int64_t end, const uint32_t* __restrict__ ent,
                                                   const uint16_t* __restrict__ vidx, int vbits, const double2* tab,
                                                   const double2* __restrict__ X, int64_t ldx_, int col0, int k,
                                                   double2* acc) {
    constexpr int SLOTS = Slots<KW>::N;
    const int lane = threadIdx.x & 31;
    const int slot = lane / KW;
    const int c = lane % KW;
    const bool slot_ok = slot < SLOTS;
    const uint32_t vmask = WIDE ? 0u : (1u << vbits) - 1u;
    bool colok[TG];
#pragma unroll
    for (int g = 0; g < TG; ++g) {
        colok[g] = slot_ok && (col0 + g * KW + c < k);
        acc[g] = make_double2(0.0, 0.0);
    }
    if (SLOTS == 1) {
        auto one = [&](int64_t j) {
            int64_t cc;
            uint32_t vi;
            pk_decode<WIDE>(ld_stream1(ent + j), WIDE ? ld_stream_u16(vidx + j) : 0u, vbits, vmask, cc, vi);
            const double2 v = tab[vi];
#pragma unroll
            for (int g = 0; g < TG; ++g)
                if (colok[g]) acc[g] = fma_c(v, ldx(X + cc * ldx_ + col0 + g * KW + c), acc[g]);
        };
        int64_t j = start;
        for (; j < end && (j & 3); ++j) one(j);
        // narrow form: the next batch's words load while this batch's gathers run (4 % faster
        // on 768 columns).  Not in the wide form: its extra index registers push it past the
        // 64-register cap into spills inside this loop (1.7x slower on 10 M rows).
        uint4 w4n = (!WIDE && j + 4 <= end) ? ld_stream4(ent + j) : make_uint4(0u, 0u, 0u, 0u);
        for (; j + 4 <= end; j += 4) {
            uint4 w4;
            uint2 i4;
            if constexpr (WIDE) {
                w4 = ld_stream4(ent + j);
                i4 = ld_stream_u16x4(vidx + j);
            } else {
                w4 = w4n;
                if (j + 8 <= end) w4n = ld_stream4(ent + j + 4);
            }
            const uint32_t w[4] = {w4.x, w4.y, w4.z, w4.w};
            uint32_t vi[4] = {0u, 0u, 0u, 0u};
            if constexpr (WIDE) {
                vi[0] = i4.x & 0xffffu;
                vi[1] = i4.x >> 16;
                vi[2] = i4.y & 0xffffu;
                vi[3] = i4.y >> 16;
            }
            double2 v[4], xs[4][TG];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                int64_t cc;
                uint32_t q;
                pk_decode<WIDE>(w[u], vi[u], vbits, vmask, cc, q);
                v[u] = tab[q];
#pragma unroll
                for (int g = 0; g < TG; ++g)
                    xs[u][g] = colok[g] ? ldx(X + cc * ldx_ + col0 + g * KW + c) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int g = 0; g < TG; ++g) acc[g] = fma_c(v[u], xs[u][g], acc[g]);
        }
        for (; j < end; ++j) one(j);
    } else {
        constexpr int U = 4;
        // words of the next U groups load while this batch's gathers run
        uint32_t nw[U], ni[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t j = start + (int64_t)u * SLOTS + slot;
            const bool ok = slot_ok && j < end;
            nw[u] = ok ? ld_stream1(ent + j) : 0u;
            ni[u] = (WIDE && ok) ? ld_stream_u16(vidx + j) : 0u;
        }
        for (int64_t base = start; base < end; base += (int64_t)SLOTS * U) {
            uint32_t w[U], wi[U];
            bool ok[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t j = base + (int64_t)u * SLOTS + slot;
                ok[u] = slot_ok && j < end;
                w[u] = nw[u];
                wi[u] = ni[u];
                const int64_t jn = j + (int64_t)SLOTS * U;
                const bool okn = slot_ok && jn < end;
                nw[u] = okn ? ld_stream1(ent + jn) : 0u;
                ni[u] = (WIDE && okn) ? ld_stream_u16(vidx + jn) : 0u;
            }
            double2 v[U], xs[U][TG];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                int64_t cc;
                uint32_t q;
                pk_decode<WIDE>(w[u], wi[u], vbits, vmask, cc, q);
                v[u] = ok[u] ? tab[q] : make_double2(0.0, 0.0);
#pragma unroll
                for (int g = 0; g < TG; ++g)
                    xs[u][g] = (ok[u] && colok[g]) ? ldx(X + cc * ldx_ + col0 + g * KW + c) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int g = 0; g < TG; ++g) acc[g] = fma_c(v[u], xs[u][g], acc[g]);
        }
    }
#pragma unroll
    for (int g = 0; g < TG; ++g) {
        if (Slots<KW>::POW2) {
#pragma unroll
            for (int off = KW; off < 32; off <<= 1) acc[g] = xor_sum(acc[g], off);
        } else {
            double2 tot = make_double2(0.0, 0.0);
#pragma unroll
            for (int s = 0; s < SLOTS; ++s) {
                double2 o;
                o.x = __shfl_sync(0xffffffffu, acc[g].x, s * KW + c);
                o.y = __shfl_sync(0xffffffffu, acc[g].y, s * KW + c);
                tot = add_c(tot, o);
            }
            acc[g] = tot;
        }
    }
}

}  // namespace edx
