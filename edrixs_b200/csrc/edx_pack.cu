// edx_pack.cu -- packed form of a square complex128 matrix: dense diagonal, and per
// off-diagonal entry its column and an index into the table of distinct values, either in
// one 32-bit word (column << vbits | index) or, for matrices with too many columns for that,
// as a 32-bit column plus a 16-bit index.
//
// Count pass: split diagonal / off-diagonal (CSR order kept) in row chunks of at most 2^26
// off-diagonal entries; per chunk, sort the value bit patterns lexicographically (two stable
// radix sorts: imaginary bits, then real bits), flag the first of every run of equal patterns
// and scan the flags: the chunk's distinct values in ascending bit order.  The host merges
// the chunks' tables.  Fill pass: every entry finds its value in the table by binary search
// over the same bit patterns, so values are carried bit for bit.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <utility>
#include <vector>

#include "edx_common.cuh"

namespace edx {

int check_csr(const edx_csr* A);

namespace {

__device__ __forceinline__ uint64_t bits_of(double v) { return (uint64_t)__double_as_longlong(v); }

// off-diagonal entries per row (the CSR holds at most one diagonal entry per row)
__global__ void k_pk_count(int64_t n, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                           int64_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t ws = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = w0; r < n; r += ws) {
        const int64_t s = row_ptr[r], e = row_ptr[r + 1];
        int d = 0;
        for (int64_t j = s + lane; j < e; j += 32) d += (col[j] == r);
        d = __reduce_add_sync(0xffffffffu, d);
        if (lane == 0) cnt[r] = (e - s) - d;
    }
}

// rows [r0, r1): diagonal into diag, off-diagonal value bits (re, im) into the key arrays at
// off_ptr[r] - base + i
__global__ void k_pk_split(int64_t r0, int64_t r1, int64_t base, const int64_t* __restrict__ row_ptr,
                           const int32_t* __restrict__ col, const double2* __restrict__ val,
                           const int64_t* __restrict__ off_ptr, double2* __restrict__ diag, uint64_t* __restrict__ re,
                           uint64_t* __restrict__ im) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t ws = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = r0 + w0; r < r1; r += ws) {
        const int64_t s = row_ptr[r], e = row_ptr[r + 1];
        int64_t o = off_ptr[r] - base;
        double2 dg = make_double2(0.0, 0.0);
        for (int64_t b = s; b < e; b += 32) {
            const int64_t j = b + lane;
            const bool in = j < e;
            const bool isd = in && col[j] == r;
            const bool off = in && !isd;
            const double2 v = in ? val[j] : make_double2(0.0, 0.0);
            const unsigned md = __ballot_sync(0xffffffffu, isd);
            if (md) dg = shfl2(v, __ffs(md) - 1);
            const unsigned m = __ballot_sync(0xffffffffu, off);
            if (off) {
                const int64_t q = o + __popc(m & ((1u << lane) - 1u));
                re[q] = bits_of(v.x);
                im[q] = bits_of(v.y);
            }
            o += __popc(m);
        }
        if (lane == 0) diag[r] = dg;
    }
}

__global__ void k_pk_flags(int64_t m, const uint64_t* __restrict__ re, const uint64_t* __restrict__ im,
                           int32_t* __restrict__ flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || re[i] != re[i - 1] || im[i] != im[i - 1]) ? 1 : 0;
}

__global__ void k_pk_table(int64_t m, const uint64_t* __restrict__ re, const uint64_t* __restrict__ im,
                           const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                           uint64_t* __restrict__ tre, uint64_t* __restrict__ tim, int32_t* __restrict__ count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (flag[i] && pos[i] < EDX_PACK_VALUES_MAX) {
            tre[pos[i]] = re[i];
            tim[pos[i]] = im[i];
        }
        if (i == m - 1) *count = pos[i] + flag[i];
    }
}

// warp per row: pack every off-diagonal entry; the value index by binary search in the table
// (narrow form: one word; wide form, vbits == 0: column word + 16-bit index)
__global__ void k_pk_fill(int64_t n, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                          const double2* __restrict__ val, const int64_t* __restrict__ off_ptr,
                          const uint64_t* __restrict__ tre, const uint64_t* __restrict__ tim, int nval, int vbits,
                          uint32_t* __restrict__ ent, uint16_t* __restrict__ vidx) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t ws = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = w0; r < n; r += ws) {
        const int64_t s = row_ptr[r], e = row_ptr[r + 1];
        int64_t o = off_ptr[r];
        for (int64_t base = s; base < e; base += 32) {
            const int64_t j = base + lane;
            const bool off = j < e && col[j] != r;
            const unsigned m = __ballot_sync(0xffffffffu, off);
            if (off) {
                const double2 v = val[j];
                const uint64_t a = bits_of(v.x), b = bits_of(v.y);
                int lo = 0, hi = nval - 1;
                while (lo < hi) {  // first table slot >= (a, b)
                    const int mid = (lo + hi) >> 1;
                    const uint64_t ta = tre[mid], tb = tim[mid];
                    if (ta < a || (ta == a && tb < b)) lo = mid + 1;
                    else hi = mid;
                }
                const int64_t q = o + __popc(m & ((1u << lane) - 1u));
                if (vbits > 0) {
                    ent[q] = ((uint32_t)col[j] << vbits) | (uint32_t)lo;
                } else {
                    ent[q] = (uint32_t)col[j];
                    vidx[q] = (uint16_t)lo;
                }
            }
            o += __popc(m);
        }
    }
}

__global__ void k_pk_vals(int nval, const uint64_t* __restrict__ tre, const uint64_t* __restrict__ tim,
                          double2* __restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nval) vals[i] = make_double2(__longlong_as_double((long long)tre[i]), __longlong_as_double((long long)tim[i]));
}

struct PackWs {
    int64_t *cnt, *off_ptr;
    double2* diag;
    uint64_t *re0, *im0, *re1, *im1, *tre, *tim;
    int32_t *flag, *pos, *count;
    void* temp;
    size_t temp_bytes;
};

// off-diagonal entries sorted at once by the count pass
constexpr int64_t PACK_CHUNK = (int64_t)1 << 26;

int64_t chunk_entries(int64_t nnz) { return std::max<int64_t>(1, std::min<int64_t>(nnz, PACK_CHUNK)); }

int pack_temp_bytes(int64_t n, int64_t nnz, size_t* out) {
    const int ch = (int)chunk_entries(nnz);
    size_t a = 0, b = 0, c = 0;
    EDX_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, a, (const int64_t*)nullptr, (int64_t*)nullptr, (int)(n + 1)));
    EDX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                             (const uint64_t*)nullptr, (uint64_t*)nullptr, ch));
    EDX_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c, (const int32_t*)nullptr, (int32_t*)nullptr, ch));
    *out = std::max(a, std::max(b, c));
    return EDX_OK;
}

template <class WS>
void pack_layout(WS& w, int64_t n, int64_t nnz, size_t temp, PackWs* o) {
    const size_t ch = (size_t)chunk_entries(nnz);
    auto cnt = w.template take<int64_t>((size_t)n + 1);
    auto off = w.template take<int64_t>((size_t)n + 1);
    auto dg = w.template take<double2>((size_t)n);
    auto re0 = w.template take<uint64_t>(ch);
    auto im0 = w.template take<uint64_t>(ch);
    auto re1 = w.template take<uint64_t>(ch);
    auto im1 = w.template take<uint64_t>(ch);
    auto fl = w.template take<int32_t>(ch);
    auto ps = w.template take<int32_t>(ch);
    auto tre = w.template take<uint64_t>(EDX_PACK_VALUES_MAX);
    auto tim = w.template take<uint64_t>(EDX_PACK_VALUES_MAX);
    auto ct = w.template take<int32_t>(4);  // [0] nval, [1] vbits (0 = wide)
    auto tmp = w.template take<char>(temp);
    if (o) *o = PackWs{cnt, off, dg, re0, im0, re1, im1, tre, tim, fl, ps, ct, tmp, temp};
}

struct SizeOnlyP {
    WorkspaceSize s;
    template <class T>
    T* take(size_t c) {
        s.take<T>(c);
        return nullptr;
    }
};

int check_square(const edx_csr* A) {
    int rc = check_csr(A);
    if (rc) return rc;
    EDX_REQUIRE(A->nrows == A->ncols && A->nrows >= 1, "edx_pack: matrix must be square and non-empty");
    EDX_REQUIRE(A->val_type == EDX_C128, "edx_pack: complex128 matrices only");
    EDX_REQUIRE(A->nnz >= 1, "edx_pack: the matrix has no entries");
    return EDX_OK;
}

int value_bits(int64_t ncols) {
    int cb = 1;
    while (cb < 32 && ((int64_t)1 << cb) < ncols) ++cb;
    return 32 - cb;
}

// row chunks [b[i], b[i+1]) holding at most PACK_CHUNK off-diagonal entries each
int row_chunks(const int64_t* d_off, int64_t n, int64_t m, std::vector<int64_t>* b, cudaStream_t st) {
    b->assign(1, 0);
    if (m <= PACK_CHUNK) {
        b->push_back(n);
        return EDX_OK;
    }
    std::vector<int64_t> off((size_t)n + 1);
    EDX_CUDA(cudaMemcpyAsync(off.data(), d_off, sizeof(int64_t) * (size_t)(n + 1), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    int64_t r0 = 0;
    while (r0 < n) {
        // last r1 with off[r1] - off[r0] <= PACK_CHUNK
        const int64_t lim = off[(size_t)r0] + PACK_CHUNK;
        int64_t r1 = (int64_t)(std::upper_bound(off.begin() + r0, off.end(), lim) - off.begin()) - 1;
        if (r1 <= r0)
            return fail(EDX_ERR_INVALID, "edx_pack_count: row %lld has more than %lld entries", (long long)r0,
                        (long long)PACK_CHUNK);
        b->push_back(r1);
        r0 = r1;
    }
    return EDX_OK;
}

}  // namespace
}  // namespace edx

using namespace edx;

extern "C" int edx_pack_workspace(const edx_csr* A, size_t* bytes) {
    int rc = check_square(A);
    if (rc) return rc;
    EDX_REQUIRE(bytes, "edx_pack_workspace: bytes missing");
    size_t temp = 0;
    if ((rc = pack_temp_bytes(A->nrows, A->nnz, &temp))) return rc;
    SizeOnlyP s;
    pack_layout(s, A->nrows, A->nnz, temp, nullptr);
    *bytes = s.s.bytes();
    return EDX_OK;
}

extern "C" int edx_pack_count(const edx_csr* A, int form, int64_t* nnz_off, int* nval, int* vbits, void* d_work,
                              size_t work_bytes, void* stream) {
    int rc = check_square(A);
    if (rc) return rc;
    EDX_REQUIRE(nnz_off && nval && vbits, "edx_pack_count: output pointers missing");
    EDX_REQUIRE(form == EDX_PACK_AUTO || form == EDX_PACK_NARROW || form == EDX_PACK_WIDE,
                "edx_pack_count: form must be EDX_PACK_AUTO, _NARROW or _WIDE");
    cudaStream_t st = as_stream(stream);
    const int64_t n = A->nrows;
    size_t temp = 0;
    if ((rc = pack_temp_bytes(n, A->nnz, &temp))) return rc;
    Workspace w(d_work, work_bytes);
    PackWs p;
    pack_layout(w, n, A->nnz, temp, &p);
    if (!p.temp) return fail(EDX_ERR_WORKSPACE, "edx_pack_count: workspace too small");
    const int grid = num_sms() * 8;
    EDX_CUDA(cudaMemsetAsync(p.cnt + n, 0, sizeof(int64_t), st));
    k_pk_count<<<grid, 256, 0, st>>>(n, A->row_ptr, A->col, p.cnt);
    EDX_CHECK_LAUNCH();
    size_t tb = p.temp_bytes;
    EDX_CUDA(cub::DeviceScan::ExclusiveSum(p.temp, tb, p.cnt, p.off_ptr, (int)(n + 1), st));
    int64_t m = 0;
    EDX_CUDA(cudaMemcpyAsync(&m, p.off_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    std::vector<int64_t> bounds;
    if ((rc = row_chunks(p.off_ptr, n, m, &bounds, st))) return rc;
    // distinct values of every chunk, merged on the host in ascending (re, im) bit order
    std::vector<std::pair<uint64_t, uint64_t>> table;
    std::vector<uint64_t> hre(EDX_PACK_VALUES_MAX), him(EDX_PACK_VALUES_MAX);
    for (size_t c = 0; c + 1 < bounds.size(); ++c) {
        const int64_t r0 = bounds[c], r1 = bounds[c + 1];
        int64_t o[2] = {0, 0};
        EDX_CUDA(cudaMemcpyAsync(&o[0], p.off_ptr + r0, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        EDX_CUDA(cudaMemcpyAsync(&o[1], p.off_ptr + r1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        EDX_CUDA(cudaStreamSynchronize(st));
        const int64_t mc = o[1] - o[0];
        k_pk_split<<<grid, 256, 0, st>>>(r0, r1, o[0], A->row_ptr, A->col, reinterpret_cast<const double2*>(A->val),
                                         p.off_ptr, p.diag, p.re0, p.im0);
        EDX_CHECK_LAUNCH();
        if (mc == 0) continue;
        // lexicographic (re, im): stable sort by im, then stable sort by re
        tb = p.temp_bytes;
        EDX_CUDA(cub::DeviceRadixSort::SortPairs(p.temp, tb, p.im0, p.im1, p.re0, p.re1, (int)mc, 0, 64, st));
        tb = p.temp_bytes;
        EDX_CUDA(cub::DeviceRadixSort::SortPairs(p.temp, tb, p.re1, p.re0, p.im1, p.im0, (int)mc, 0, 64, st));
        k_pk_flags<<<grid, 256, 0, st>>>(mc, p.re0, p.im0, p.flag);
        EDX_CHECK_LAUNCH();
        tb = p.temp_bytes;
        EDX_CUDA(cub::DeviceScan::ExclusiveSum(p.temp, tb, p.flag, p.pos, (int)mc, st));
        k_pk_table<<<grid, 256, 0, st>>>(mc, p.re0, p.im0, p.flag, p.pos, p.tre, p.tim, p.count);
        EDX_CHECK_LAUNCH();
        int cc = 0;
        EDX_CUDA(cudaMemcpyAsync(&cc, p.count, sizeof(int), cudaMemcpyDeviceToHost, st));
        EDX_CUDA(cudaStreamSynchronize(st));
        if (cc > EDX_PACK_VALUES_MAX)
            return fail(EDX_ERR_OVERFLOW, "edx_pack_count: more than %d distinct off-diagonal values",
                        EDX_PACK_VALUES_MAX);
        EDX_CUDA(cudaMemcpyAsync(hre.data(), p.tre, sizeof(uint64_t) * (size_t)cc, cudaMemcpyDeviceToHost, st));
        EDX_CUDA(cudaMemcpyAsync(him.data(), p.tim, sizeof(uint64_t) * (size_t)cc, cudaMemcpyDeviceToHost, st));
        EDX_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < cc; ++i) table.emplace_back(hre[(size_t)i], him[(size_t)i]);
        std::sort(table.begin(), table.end());
        table.erase(std::unique(table.begin(), table.end()), table.end());
        if ((int64_t)table.size() > EDX_PACK_VALUES_MAX)
            return fail(EDX_ERR_OVERFLOW, "edx_pack_count: more than %d distinct off-diagonal values",
                        EDX_PACK_VALUES_MAX);
    }
    const int count = (int)table.size();
    const int vb = value_bits(A->ncols);
    const bool narrow_fits = count <= ((int64_t)1 << vb);
    int vsel;
    if (form == EDX_PACK_NARROW) {
        if (!narrow_fits)
            return fail(EDX_ERR_OVERFLOW,
                        "edx_pack_count: %d distinct off-diagonal values, at most %lld fit the 32-bit word", count,
                        (long long)((int64_t)1 << vb));
        vsel = vb;
    } else if (form == EDX_PACK_WIDE) {
        vsel = 0;
    } else {
        vsel = narrow_fits ? vb : 0;
    }
    for (int i = 0; i < count; ++i) {
        hre[(size_t)i] = table[(size_t)i].first;
        him[(size_t)i] = table[(size_t)i].second;
    }
    if (count > 0) {
        EDX_CUDA(cudaMemcpyAsync(p.tre, hre.data(), sizeof(uint64_t) * (size_t)count, cudaMemcpyHostToDevice, st));
        EDX_CUDA(cudaMemcpyAsync(p.tim, him.data(), sizeof(uint64_t) * (size_t)count, cudaMemcpyHostToDevice, st));
    }
    const int32_t hc[2] = {count, vsel};
    EDX_CUDA(cudaMemcpyAsync(p.count, hc, sizeof(hc), cudaMemcpyHostToDevice, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    *nnz_off = m;
    *nval = count;
    *vbits = vsel;
    return EDX_OK;
}

extern "C" int edx_pack_fill(const edx_csr* A, edx_packed* P, void* d_work, size_t work_bytes, void* stream) {
    int rc = check_square(A);
    if (rc) return rc;
    EDX_REQUIRE(P && P->row_ptr && P->diag && (P->nnz == 0 || (P->ent && P->vals && P->nval >= 1)),
                "edx_pack_fill: output arrays missing");
    EDX_REQUIRE(P->vbits > 0 || P->nnz == 0 || P->vidx, "edx_pack_fill: the wide form needs vidx");
    cudaStream_t st = as_stream(stream);
    const int64_t n = A->nrows;
    size_t temp = 0;
    if ((rc = pack_temp_bytes(n, A->nnz, &temp))) return rc;
    Workspace w(d_work, work_bytes);
    PackWs p;
    pack_layout(w, n, A->nnz, temp, &p);
    if (!p.temp) return fail(EDX_ERR_WORKSPACE, "edx_pack_fill: workspace too small");
    int64_t m = 0;
    int32_t hc[2] = {0, 0};
    EDX_CUDA(cudaMemcpyAsync(&m, p.off_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaMemcpyAsync(hc, p.count, sizeof(hc), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    EDX_REQUIRE(m == P->nnz && hc[0] == P->nval && hc[1] == P->vbits,
                "edx_pack_fill: sizes differ from the count pass");
    P->nrows = n;
    EDX_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(P->row_ptr), p.off_ptr, sizeof(int64_t) * (size_t)(n + 1),
                             cudaMemcpyDeviceToDevice, st));
    EDX_CUDA(cudaMemcpyAsync(const_cast<double*>(P->diag), p.diag, sizeof(double2) * (size_t)n,
                             cudaMemcpyDeviceToDevice, st));
    if (m > 0) {
        k_pk_vals<<<(hc[0] + 127) / 128, 128, 0, st>>>(hc[0], p.tre, p.tim,
                                                       reinterpret_cast<double2*>(const_cast<double*>(P->vals)));
        EDX_CHECK_LAUNCH();
        k_pk_fill<<<num_sms() * 8, 256, 0, st>>>(n, A->row_ptr, A->col, reinterpret_cast<const double2*>(A->val),
                                                 p.off_ptr, p.tre, p.tim, hc[0], P->vbits,
                                                 const_cast<uint32_t*>(P->ent), const_cast<uint16_t*>(P->vidx));
        EDX_CHECK_LAUNCH();
    }
    return EDX_OK;
}
