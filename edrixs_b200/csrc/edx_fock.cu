// edx_fock.cu -- error state, device queries and the Fock-basis kernels (K1 unrank, K2 rank).
//
// A Fock state is a 64-bit word: orbital p (1-based in the files) is bit p-1
// (src/fock.f90:52-61).  The full N-electron sector of norb orbitals in ascending integer
// order is exactly the colex order of N-subsets, so state i is the i-th subset of the
// combinatorial number system: i = sum_j C(c_j, j) over the set bits c_1 < ... < c_N
// (j = 1..N).  Unranking inverts that sum greedily from the top bit.
#include <cstring>
#include <mutex>
#include <vector>

#include "edx_common.cuh"
#include "edx_fock.cuh"

namespace edx {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int num_sms() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

uint64_t host_binomial(int n, int k) {
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (int i = 1; i <= k; ++i) r = r * (unsigned)(n - k + i) / (unsigned)i;
    return (uint64_t)r;
}

// ---- kernels -------------------------------------------------------------------------

__global__ void k_fock_unrank(int norb, int nelec, uint64_t* __restrict__ fock, int64_t ndim) {
    extern __shared__ uint64_t tab[];
    binom_fill(tab, norb, nelec);
    __syncthreads();
    const int kk = nelec + 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ndim;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t r = (uint64_t)i, s = 0;
        int c = norb - 1;
        for (int j = nelec; j >= 1; --j) {
            // largest c with C(c, j) <= r
            while (c >= j && tab[c * kk + j] > r) --c;
            if (c < j - 1) c = j - 1;
            s |= 1ull << c;
            r -= tab[c * kk + j];
            --c;
        }
        fock[i] = s;
    }
}

__global__ void k_fock_match(int norb, int nelec, const uint64_t* __restrict__ fock, int64_t ndim,
                             int* mismatch) {
    extern __shared__ uint64_t tab[];
    binom_fill(tab, norb, nelec);
    __syncthreads();
    int bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ndim;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = fock_rank(tab, norb, nelec, fock[i]);
        if (r != i) bad = 1;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(mismatch, 1);
}

}  // namespace edx

using namespace edx;

extern "C" const char* edx_last_error(void) { return g_err.c_str(); }
extern "C" int edx_abi_version(void) { return EDX_ABI_VERSION; }

extern "C" int edx_fock_count(int norb, int nelec, int64_t* ndim) {
    EDX_REQUIRE(ndim != nullptr, "edx_fock_count: ndim is NULL");
    EDX_REQUIRE(norb >= 0 && norb <= 63 && nelec >= 0 && nelec <= norb,
                "edx_fock_count: need 0 <= nelec <= norb <= 63 (got norb=%d nelec=%d)", norb, nelec);
    *ndim = (int64_t)host_binomial(norb, nelec);
    return EDX_OK;
}

extern "C" int edx_fock_unrank(int norb, int nelec, uint64_t* d_fock, int64_t ndim, void* stream) {
    EDX_REQUIRE(norb >= 1 && norb <= 63 && nelec >= 0 && nelec <= norb,
                "edx_fock_unrank: need 0 <= nelec <= norb <= 63 (got norb=%d nelec=%d)", norb, nelec);
    int64_t want = (int64_t)host_binomial(norb, nelec);
    EDX_REQUIRE(ndim == want, "edx_fock_unrank: ndim=%lld but C(%d,%d)=%lld", (long long)ndim, norb,
                nelec, (long long)want);
    EDX_REQUIRE(d_fock != nullptr || ndim == 0, "edx_fock_unrank: d_fock is NULL");
    if (ndim == 0) return EDX_OK;
    size_t smem = binom_bytes(norb, nelec);
    int threads = 256;
    int64_t blocks = (ndim + threads - 1) / threads;
    int maxb = num_sms() * 8;
    if (blocks > maxb) blocks = maxb;
    k_fock_unrank<<<(unsigned)blocks, threads, smem, as_stream(stream)>>>(norb, nelec, d_fock, ndim);
    EDX_CHECK_LAUNCH();
    return EDX_OK;
}

extern "C" int edx_fock_match_full_workspace(size_t* bytes) {
    EDX_REQUIRE(bytes != nullptr, "NULL bytes");
    *bytes = 256;
    return EDX_OK;
}

extern "C" int edx_fock_match_full(int norb, int nelec, const uint64_t* d_fock, int64_t ndim,
                                   int* is_full, void* d_work, size_t work_bytes, void* stream) {
    EDX_REQUIRE(is_full != nullptr, "edx_fock_match_full: is_full is NULL");
    *is_full = 0;
    if (norb < 1 || norb > 63 || nelec < 0 || nelec > norb) return EDX_OK;
    if ((int64_t)host_binomial(norb, nelec) != ndim || ndim == 0) return EDX_OK;
    Workspace ws(d_work, work_bytes);
    int* flag = ws.take<int>(1);
    if (!flag) return fail(EDX_ERR_WORKSPACE, "edx_fock_match_full: workspace too small");
    cudaStream_t st = as_stream(stream);
    EDX_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
    int threads = 256;
    int64_t blocks = (ndim + threads - 1) / threads;
    int maxb = num_sms() * 8;
    if (blocks > maxb) blocks = maxb;
    k_fock_match<<<(unsigned)blocks, threads, binom_bytes(norb, nelec), st>>>(norb, nelec, d_fock,
                                                                            ndim, flag);
    EDX_CHECK_LAUNCH();
    int h = 1;
    EDX_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    EDX_CUDA(cudaStreamSynchronize(st));
    *is_full = (h == 0) ? 1 : 0;
    return EDX_OK;
}
