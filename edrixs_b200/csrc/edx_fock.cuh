// edx_fock.cuh -- device helpers for Fock states: binomial table, rank, fermion sign.
#pragma once
#include <stdint.h>

namespace edx {

uint64_t host_binomial(int n, int k);

// shared-memory table C(n, j) for 0 <= n <= norb, 0 <= j <= nelec+1, row-major with
// (nelec+2) columns... we keep nelec+1 columns: j in [0, nelec]
__host__ __device__ inline size_t binom_bytes(int norb, int nelec) {
    return sizeof(uint64_t) * (size_t)(norb + 1) * (size_t)(nelec + 1);
}

// Pascal's triangle, one row per step; all threads of the block participate.
__device__ inline void binom_fill(uint64_t* tab, int norb, int nelec) {
    const int kk = nelec + 1;
    for (int j = threadIdx.x; j < kk; j += blockDim.x) tab[j] = (j == 0) ? 1ull : 0ull;
    __syncthreads();
    for (int n = 1; n <= norb; ++n) {
        for (int j = threadIdx.x; j < kk; j += blockDim.x) {
            uint64_t a = tab[(n - 1) * kk + j];
            uint64_t b = (j > 0) ? tab[(n - 1) * kk + j - 1] : 0ull;
            tab[n * kk + j] = a + b;
        }
        __syncthreads();
    }
}

// 0-based rank of state s in the ascending full norb/nelec basis, or -1 if s is not in it.
__device__ inline int64_t fock_rank(const uint64_t* tab, int norb, int nelec, uint64_t s) {
    if (norb < 64 && (s >> norb) != 0ull) return -1;
    if (__popcll(s) != nelec) return -1;
    const int kk = nelec + 1;
    uint64_t r = 0;
    int j = 1;
    while (s) {
        int c = __ffsll((long long)s) - 1;
        r += tab[c * kk + j];
        s &= s - 1;
        ++j;
    }
    return (int64_t)r;
}

// binary search of src/utils.f90:2-40 on an ascending array; 0-based index or -1.
__device__ inline int64_t fock_search(const uint64_t* __restrict__ v, int64_t n, uint64_t m) {
    int64_t lo = 0, hi = n - 1;
    while (lo <= hi) {
        int64_t mid = lo + ((hi - lo) >> 1);
        uint64_t x = __ldg(reinterpret_cast<const unsigned long long*>(v) + mid);
        if (x < m) lo = mid + 1;
        else if (x > m) hi = mid - 1;
        else return mid;
    }
    return -1;
}

// parity of the occupied orbitals strictly below bit p (src/fock.f90:52-56): 1 = odd
__device__ inline int below_parity(uint64_t s, int p) {
    uint64_t mask = (p >= 64) ? ~0ull : ((1ull << p) - 1ull);
    return __popcll(s & mask) & 1;
}

}  // namespace edx
