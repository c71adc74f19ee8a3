// edx_tiles.cu -- tiled layout of a square CSR matrix: entries grouped by (row tile, column
// tile) pair, cut at row boundaries into pieces that one block stages in shared memory.
//
// Build (two passes over the same workspace):
//   1. column tile of every entry (key) and its position (value), row of every entry
//   2. stable segmented sort of (key, position) per row tile: order (column tile, row, col)
//   3. run-length encoding of (row tile, column tile) over the sorted entries = the pairs
//   4. per pair (one thread): walk its rows, cut pieces of <= EDX_TILE_PIECE_MAX entries
//      (count pass: sizes; fill pass: descriptors, headers, local columns, values)
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <vector>

#include "edx_common.cuh"

namespace edx {

int check_csr(const edx_csr* A);

namespace {

constexpr int ENT_ALIGN = 16;  // entries of a piece start on a multiple of 16 (16-byte lcol chunks)
constexpr int HDR_ALIGN = 8;   // headers of a piece start on a multiple of 8 (16-byte chunks)

__host__ __device__ inline int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

__global__ void k_tl_tile_of(int nt, const int32_t* __restrict__ start, int32_t* __restrict__ tile_of) {
    for (int t = blockIdx.x; t < nt; t += gridDim.x)
        for (int32_t i = start[t] + (int32_t)threadIdx.x; i < start[t + 1]; i += (int32_t)blockDim.x) tile_of[i] = t;
}

__global__ void k_tl_segments(int ntr, const int32_t* __restrict__ tile_r, const int64_t* __restrict__ row_ptr,
                              int32_t* __restrict__ seg) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= ntr) seg[t] = (int32_t)row_ptr[tile_r[t]];
}

// warp per row: key = column tile of the entry, value = entry position, row of the entry
__global__ void k_tl_keys(int64_t n, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                          const int32_t* __restrict__ ctile_of, int32_t* __restrict__ key, int32_t* __restrict__ pos,
                          int32_t* __restrict__ row_of) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t ws = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = w0; r < n; r += ws) {
        const int64_t e = row_ptr[r + 1];
        for (int64_t j = row_ptr[r] + lane; j < e; j += 32) {
            key[j] = ctile_of[col[j]];
            pos[j] = (int32_t)j;
            row_of[j] = (int32_t)r;
        }
    }
}

// (row tile << 32 | column tile) of every sorted entry; non-decreasing along the sorted order
__global__ void k_tl_pairkey(int32_t nnz, const int32_t* __restrict__ key_s, const int32_t* __restrict__ pos_s,
                             const int32_t* __restrict__ row_of, const int32_t* __restrict__ rtile_of,
                             uint64_t* __restrict__ pk) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
        pk[i] = ((uint64_t)(uint32_t)rtile_of[row_of[pos_s[i]]] << 32) | (uint32_t)key_s[i];
}

struct PairWalk {
    const int32_t* pos_s;
    const int32_t* row_of;
    __device__ int row(int64_t q) const { return row_of[pos_s[q]]; }
    // one past the last sorted position of the row that starts at q
    __device__ int64_t row_end(int64_t q, int64_t pend) const {
        const int r = row(q);
        int64_t q2 = q + 1;
        while (q2 < pend && row(q2) == r) ++q2;
        return q2;
    }
    // one past the last position of the piece that starts at p (whole rows, <= max entries,
    // at least one row)
    __device__ int64_t piece_end(int64_t p, int64_t pend) const {
        int64_t q = p;
        while (q < pend) {
            const int64_t q2 = row_end(q, pend);
            if (q > p && (q2 - p) > EDX_TILE_PIECE_MAX) break;
            q = q2;
        }
        return q;
    }
};

// pass 1: pieces, padded entries and padded header slots of every pair
__global__ void k_tl_count(int npairs, const int32_t* __restrict__ pair_pos, const int32_t* __restrict__ runlen,
                           PairWalk W, int64_t* __restrict__ c_piece, int64_t* __restrict__ c_ent,
                           int64_t* __restrict__ c_hdr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const int64_t p0 = pair_pos[i], pend = p0 + runlen[i];
    int64_t np = 0, ne = 0, nh = 0;
    for (int64_t p = p0; p < pend;) {
        const int64_t q = W.piece_end(p, pend);
        const int ra = W.row(p), rb = W.row(q - 1) + 1;
        ++np;
        ne += round_up(q - p, ENT_ALIGN);
        nh += round_up(rb - ra + 1, HDR_ALIGN);
        p = q;
    }
    c_piece[i] = np;
    c_ent[i] = ne;
    c_hdr[i] = nh;
}

struct TilesOut {
    int32_t* piece_ctile;
    int32_t* piece_rows;
    int64_t* piece_ent;
    int64_t* piece_hdr;
    uint16_t* hdr;
    uint8_t* lcol;
    double2* val;
};

// pass 2: one thread writes every piece of its pair
__global__ void k_tl_fill(int npairs, const uint64_t* __restrict__ uniq, const int32_t* __restrict__ pair_pos,
                          const int32_t* __restrict__ runlen, PairWalk W, const int32_t* __restrict__ tile_r,
                          const int32_t* __restrict__ tile_c, const int32_t* __restrict__ col,
                          const double2* __restrict__ val, const int64_t* __restrict__ o_piece,
                          const int64_t* __restrict__ o_ent, const int64_t* __restrict__ o_hdr, TilesOut T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const int R = (int)(uniq[i] >> 32), C = (int)(uniq[i] & 0xffffffffu);
    const int32_t rs = tile_r[R], cs = tile_c[C];
    const int64_t p0 = pair_pos[i], pend = p0 + runlen[i];
    int64_t pi = o_piece[i], e = o_ent[i], h = o_hdr[i];
    for (int64_t p = p0; p < pend;) {
        const int64_t q = W.piece_end(p, pend);
        const int ra = W.row(p), rb = W.row(q - 1) + 1;
        T.piece_ctile[pi] = C;
        T.piece_rows[pi] = (ra - rs) | ((rb - rs) << 16);
        T.piece_ent[pi] = e;
        T.piece_hdr[pi] = h;
        // hdr[h + j] = entries of rows ra .. ra+j-1 in this piece
        int cur = ra;
        T.hdr[h] = 0;
        for (int64_t t = p; t < q; ++t) {
            const int r = W.row(t);
            while (cur < r) {
                ++cur;
                T.hdr[h + (cur - ra)] = (uint16_t)(t - p);
            }
            const int32_t j = W.pos_s[t];
            T.lcol[e + (t - p)] = (uint8_t)(col[j] - cs);
            T.val[e + (t - p)] = val[j];
        }
        T.hdr[h + (rb - ra)] = (uint16_t)(q - p);
        ++pi;
        e += round_up(q - p, ENT_ALIGN);
        h += round_up(rb - ra + 1, HDR_ALIGN);
        p = q;
    }
}

// piece_ptr[R] = first piece of row tile R (pairs are in row-tile order)
__global__ void k_tl_piece_ptr(int npairs, const uint64_t* __restrict__ uniq, const int64_t* __restrict__ o_piece,
                               int32_t* __restrict__ piece_ptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npairs) return;
    const int R = (int)(uniq[i] >> 32);
    if (i == 0 || (int)(uniq[i - 1] >> 32) != R) piece_ptr[R] = (int32_t)o_piece[i];
}

// row tiles without entries take the start of the next row tile; closes both pointer arrays
__global__ void k_tl_close(int ntr, int64_t npiece, int64_t nent, int32_t* __restrict__ piece_ptr,
                           int64_t* __restrict__ piece_ent) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    piece_ptr[ntr] = (int32_t)npiece;
    for (int R = ntr - 1; R >= 0; --R)
        if (piece_ptr[R] < 0) piece_ptr[R] = piece_ptr[R + 1];
    piece_ent[npiece] = nent;
}

struct TilesWs {
    int32_t *ctile_of, *rtile_of, *seg, *key, *pos, *key_s, *pos_s, *row_of, *runlen, *pair_pos, *nruns;
    uint64_t *pk, *uniq;
    int64_t *c_piece, *c_ent, *c_hdr, *o_piece, *o_ent, *o_hdr;
    void* temp;
    size_t temp_bytes;
};

int64_t max_pairs(int64_t nnz, int32_t ntr, int32_t ntc) { return std::max<int64_t>(1, std::min<int64_t>(nnz, (int64_t)ntr * ntc)); }

// CUB scratch of the three device-wide steps (the largest of them)
int cub_temp_bytes(int32_t nnz, int32_t ntr, int64_t P, size_t* out) {
    size_t a = 0, b = 0, c = 0, d = 0;
    EDX_CUDA(cub::DeviceSegmentedSort::StableSortPairs(nullptr, a, (const int32_t*)nullptr, (int32_t*)nullptr,
                                                       (const int32_t*)nullptr, (int32_t*)nullptr, (int)nnz, (int)ntr,
                                                       (const int32_t*)nullptr, (const int32_t*)nullptr + 1));
    EDX_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, b, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                                (int32_t*)nullptr, (int32_t*)nullptr, (int)nnz));
    EDX_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c, (const int32_t*)nullptr, (int32_t*)nullptr, (int)P));
    EDX_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, d, (const int64_t*)nullptr, (int64_t*)nullptr, (int)P));
    *out = std::max(std::max(a, b), std::max(c, d));
    return EDX_OK;
}

template <class WS>
void tiles_layout(WS& w, int64_t n, int64_t nnz, int32_t ntr, int64_t P, size_t temp, TilesWs* o) {
    auto ctile_of = w.template take<int32_t>((size_t)n);
    auto rtile_of = w.template take<int32_t>((size_t)n);
    auto seg = w.template take<int32_t>((size_t)ntr + 1);
    // key and pos are dead once sorted; the pair keys reuse their bytes
    auto kp = w.template take<uint64_t>((size_t)nnz);
    auto key_s = w.template take<int32_t>((size_t)nnz);
    auto pos_s = w.template take<int32_t>((size_t)nnz);
    auto row_of = w.template take<int32_t>((size_t)nnz);
    auto uniq = w.template take<uint64_t>((size_t)P);
    auto runlen = w.template take<int32_t>((size_t)P);
    auto pair_pos = w.template take<int32_t>((size_t)P);
    auto nruns = w.template take<int32_t>(1);
    auto cnt = w.template take<int64_t>((size_t)P * 6);
    auto tmp = w.template take<char>(temp);
    if (o) {
        o->ctile_of = ctile_of;
        o->rtile_of = rtile_of;
        o->seg = seg;
        o->pk = kp;
        o->key = reinterpret_cast<int32_t*>(kp);
        o->pos = reinterpret_cast<int32_t*>(kp) + nnz;
        o->key_s = key_s;
        o->pos_s = pos_s;
        o->row_of = row_of;
        o->uniq = uniq;
        o->runlen = runlen;
        o->pair_pos = pair_pos;
        o->nruns = nruns;
        o->c_piece = cnt;
        o->c_ent = cnt ? cnt + P : nullptr;
        o->c_hdr = cnt ? cnt + 2 * P : nullptr;
        o->o_piece = cnt ? cnt + 3 * P : nullptr;
        o->o_ent = cnt ? cnt + 4 * P : nullptr;
        o->o_hdr = cnt ? cnt + 5 * P : nullptr;
        o->temp = tmp;
        o->temp_bytes = temp;
    }
}

struct SizeOnlyT {
    WorkspaceSize s;
    template <class T>
    T* take(size_t c) {
        s.take<T>(c);
        return nullptr;
    }
};

int check_tiles(const char* what, int32_t nt, const int32_t* d_start, int64_t n, int maxlen, cudaStream_t st) {
    EDX_REQUIRE(nt >= 1 && d_start, "edx_tiles: %s tiles missing", what);
    std::vector<int32_t> h((size_t)nt + 1);
    EDX_CUDA(cudaMemcpyAsync(h.data(), d_start, sizeof(int32_t) * h.size(), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    EDX_REQUIRE(h[0] == 0 && h[nt] == n, "edx_tiles: %s tiles must start at 0 and end at %lld", what, (long long)n);
    for (int32_t t = 0; t < nt; ++t) {
        const int32_t len = h[t + 1] - h[t];
        EDX_REQUIRE(len >= 1 && len <= maxlen, "edx_tiles: %s tile %d has %d indices (1..%d allowed)", what, t, len,
                    maxlen);
    }
    return EDX_OK;
}

int check_matrix(const edx_csr* A) {
    int rc = check_csr(A);
    if (rc) return rc;
    EDX_REQUIRE(A->nrows == A->ncols && A->nrows >= 1, "edx_tiles: matrix must be square and non-empty");
    EDX_REQUIRE(A->val_type == EDX_C128, "edx_tiles: complex128 matrices only");
    EDX_REQUIRE(A->nnz >= 1 && A->nnz < ((int64_t)1 << 31) && A->nrows < ((int64_t)1 << 31),
                "edx_tiles: nnz must be 1 .. 2^31-1");
    return EDX_OK;
}

// steps 1-3 and the per-pair counts + offsets; leaves everything in the workspace
int tiles_prepare(const edx_csr* A, int32_t ntr, const int32_t* tile_r, int32_t ntc, const int32_t* tile_c,
                  const TilesWs& w, int* npairs_out, cudaStream_t st) {
    const int64_t n = A->nrows;
    const int32_t nnz = (int32_t)A->nnz;
    const int sms = num_sms();
    k_tl_tile_of<<<std::min(ntc, sms * 16), 128, 0, st>>>(ntc, tile_c, w.ctile_of);
    EDX_CHECK_LAUNCH();
    k_tl_tile_of<<<std::min(ntr, sms * 16), 128, 0, st>>>(ntr, tile_r, w.rtile_of);
    EDX_CHECK_LAUNCH();
    k_tl_segments<<<(ntr + 1 + 255) / 256, 256, 0, st>>>(ntr, tile_r, A->row_ptr, w.seg);
    EDX_CHECK_LAUNCH();
    k_tl_keys<<<sms * 8, 256, 0, st>>>(n, A->row_ptr, A->col, w.ctile_of, w.key, w.pos, w.row_of);
    EDX_CHECK_LAUNCH();
    size_t tb = w.temp_bytes;
    EDX_CUDA(cub::DeviceSegmentedSort::StableSortPairs(w.temp, tb, w.key, w.key_s, w.pos, w.pos_s, (int)nnz, (int)ntr,
                                                       w.seg, w.seg + 1, st));
    k_tl_pairkey<<<sms * 8, 256, 0, st>>>(nnz, w.key_s, w.pos_s, w.row_of, w.rtile_of, w.pk);
    EDX_CHECK_LAUNCH();
    tb = w.temp_bytes;
    EDX_CUDA(cub::DeviceRunLengthEncode::Encode(w.temp, tb, w.pk, w.uniq, w.runlen, w.nruns, (int)nnz, st));
    int npairs = 0;
    EDX_CUDA(cudaMemcpyAsync(&npairs, w.nruns, sizeof(int), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    EDX_REQUIRE(npairs >= 1 && npairs <= max_pairs(nnz, ntr, ntc), "edx_tiles: bad pair count %d", npairs);
    tb = w.temp_bytes;
    EDX_CUDA(cub::DeviceScan::ExclusiveSum(w.temp, tb, w.runlen, w.pair_pos, npairs, st));
    PairWalk W{w.pos_s, w.row_of};
    k_tl_count<<<(npairs + 127) / 128, 128, 0, st>>>(npairs, w.pair_pos, w.runlen, W, w.c_piece, w.c_ent, w.c_hdr);
    EDX_CHECK_LAUNCH();
    for (int q = 0; q < 3; ++q) {
        const int64_t* in = q == 0 ? w.c_piece : (q == 1 ? w.c_ent : w.c_hdr);
        int64_t* out = q == 0 ? w.o_piece : (q == 1 ? w.o_ent : w.o_hdr);
        tb = w.temp_bytes;
        EDX_CUDA(cub::DeviceScan::ExclusiveSum(w.temp, tb, in, out, npairs, st));
    }
    *npairs_out = npairs;
    return EDX_OK;
}

int tiles_totals(const TilesWs& w, int npairs, int64_t* tot, cudaStream_t st) {
    int64_t h[6];
    const int64_t last = npairs - 1;
    EDX_CUDA(cudaMemcpyAsync(h + 0, w.o_piece + last, 8, cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaMemcpyAsync(h + 1, w.c_piece + last, 8, cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaMemcpyAsync(h + 2, w.o_ent + last, 8, cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaMemcpyAsync(h + 3, w.c_ent + last, 8, cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaMemcpyAsync(h + 4, w.o_hdr + last, 8, cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaMemcpyAsync(h + 5, w.c_hdr + last, 8, cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    tot[0] = h[0] + h[1];
    tot[1] = h[2] + h[3];
    tot[2] = h[4] + h[5];
    return EDX_OK;
}

}  // namespace
}  // namespace edx

using namespace edx;

extern "C" int edx_tiles_workspace(const edx_csr* A, int32_t ntile_r, int32_t ntile_c, size_t* bytes) {
    int rc = check_matrix(A);
    if (rc) return rc;
    EDX_REQUIRE(bytes && ntile_r >= 1 && ntile_c >= 1, "edx_tiles_workspace: bad arguments");
    const int64_t P = max_pairs(A->nnz, ntile_r, ntile_c);
    size_t temp = 0;
    rc = cub_temp_bytes((int32_t)A->nnz, ntile_r, P, &temp);
    if (rc) return rc;
    SizeOnlyT s;
    tiles_layout(s, A->nrows, A->nnz, ntile_r, P, temp, nullptr);
    *bytes = s.s.bytes();
    return EDX_OK;
}

extern "C" int edx_tiles_count(const edx_csr* A, int32_t ntile_r, const int32_t* d_tile_r, int32_t ntile_c,
                               const int32_t* d_tile_c, int64_t* npiece, int64_t* nent, int64_t* nhdr, void* d_work,
                               size_t work_bytes, void* stream) {
    int rc = check_matrix(A);
    if (rc) return rc;
    EDX_REQUIRE(npiece && nent && nhdr, "edx_tiles_count: output pointers missing");
    cudaStream_t st = as_stream(stream);
    if ((rc = check_tiles("row", ntile_r, d_tile_r, A->nrows, EDX_TILE_ROWS_MAX, st))) return rc;
    if ((rc = check_tiles("column", ntile_c, d_tile_c, A->ncols, EDX_TILE_COLS_MAX, st))) return rc;
    const int64_t P = max_pairs(A->nnz, ntile_r, ntile_c);
    size_t temp = 0;
    if ((rc = cub_temp_bytes((int32_t)A->nnz, ntile_r, P, &temp))) return rc;
    Workspace w(d_work, work_bytes);
    TilesWs ws;
    tiles_layout(w, A->nrows, A->nnz, ntile_r, P, temp, &ws);
    if (!ws.temp) return fail(EDX_ERR_WORKSPACE, "edx_tiles_count: workspace too small");
    int npairs = 0;
    if ((rc = tiles_prepare(A, ntile_r, d_tile_r, ntile_c, d_tile_c, ws, &npairs, st))) return rc;
    int64_t tot[3];
    if ((rc = tiles_totals(ws, npairs, tot, st))) return rc;
    EDX_REQUIRE(tot[0] < ((int64_t)1 << 31), "edx_tiles_count: too many pieces");
    *npiece = tot[0];
    *nent = tot[1];
    *nhdr = tot[2];
    return EDX_OK;
}

extern "C" int edx_tiles_fill(const edx_csr* A, edx_tiles* T, void* d_work, size_t work_bytes, void* stream) {
    int rc = check_matrix(A);
    if (rc) return rc;
    EDX_REQUIRE(T && T->tile_r && T->tile_c && T->piece_ptr && T->piece_ctile && T->piece_rows && T->piece_ent &&
                    T->piece_hdr && T->hdr && T->lcol && T->val && T->npiece >= 1,
                "edx_tiles_fill: output arrays missing");
    cudaStream_t st = as_stream(stream);
    const int64_t P = max_pairs(A->nnz, T->ntile_r, T->ntile_c);
    size_t temp = 0;
    if ((rc = cub_temp_bytes((int32_t)A->nnz, T->ntile_r, P, &temp))) return rc;
    Workspace w(d_work, work_bytes);
    TilesWs ws;
    tiles_layout(w, A->nrows, A->nnz, T->ntile_r, P, temp, &ws);
    if (!ws.temp) return fail(EDX_ERR_WORKSPACE, "edx_tiles_fill: workspace too small");
    int npairs = 0;
    EDX_CUDA(cudaMemcpyAsync(&npairs, ws.nruns, sizeof(int), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    EDX_REQUIRE(npairs >= 1 && npairs <= P, "edx_tiles_fill: workspace does not hold a count pass");
    int64_t tot[3];
    if ((rc = tiles_totals(ws, npairs, tot, st))) return rc;
    EDX_REQUIRE(tot[0] == T->npiece && tot[1] == T->nent && tot[2] == T->nhdr,
                "edx_tiles_fill: sizes differ from the count pass");
    T->nrows = A->nrows;
    TilesOut O{const_cast<int32_t*>(T->piece_ctile), const_cast<int32_t*>(T->piece_rows),
               const_cast<int64_t*>(T->piece_ent),   const_cast<int64_t*>(T->piece_hdr),
               const_cast<uint16_t*>(T->hdr),        const_cast<uint8_t*>(T->lcol),
               reinterpret_cast<double2*>(const_cast<void*>(T->val))};
    EDX_CUDA(cudaMemsetAsync(O.hdr, 0, sizeof(uint16_t) * (size_t)T->nhdr, st));
    EDX_CUDA(cudaMemsetAsync(O.lcol, 0, (size_t)T->nent, st));
    EDX_CUDA(cudaMemsetAsync(O.val, 0, sizeof(double2) * (size_t)T->nent, st));
    EDX_CUDA(cudaMemsetAsync(const_cast<int32_t*>(T->piece_ptr), 0xff, sizeof(int32_t) * ((size_t)T->ntile_r + 1), st));
    PairWalk W{ws.pos_s, ws.row_of};
    k_tl_fill<<<(npairs + 127) / 128, 128, 0, st>>>(npairs, ws.uniq, ws.pair_pos, ws.runlen, W, T->tile_r, T->tile_c,
                                                    A->col, reinterpret_cast<const double2*>(A->val), ws.o_piece,
                                                    ws.o_ent, ws.o_hdr, O);
    EDX_CHECK_LAUNCH();
    k_tl_piece_ptr<<<(npairs + 255) / 256, 256, 0, st>>>(npairs, ws.uniq, ws.o_piece,
                                                         const_cast<int32_t*>(T->piece_ptr));
    EDX_CHECK_LAUNCH();
    k_tl_close<<<1, 1, 0, st>>>(T->ntile_r, T->npiece, T->nent, const_cast<int32_t*>(T->piece_ptr), O.piece_ent);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}
