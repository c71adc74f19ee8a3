// edx_krylov.cuh -- state and reductions shared by the Lanczos kernels (edx_krylov.cu) and
// the slab product (edx_kron.cu).
#pragma once
#include "edx_common.cuh"

namespace edx {

// ---- deterministic cross-block reduction --------------------------------------------
__device__ __forceinline__ bool arrive_last(unsigned* ticket) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned total = gridDim.x * gridDim.y;
        last = (atomicAdd(ticket, 1u) == total - 1u);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ double sum_partials(const double* part, int nbx, int k, int gc) {
    double s = 0.0;
    for (int b = 0; b < nbx; ++b) s += __ldcg(part + (int64_t)b * k + gc);
    return s;
}

struct KrylovState {
    double* alpha_out;  // [k*maxn]
    double* beta_out;   // [k*maxn]
    int32_t* neff;      // [k]
    double* alpha;      // [k] current alpha
    double* beta;       // [k] current beta (beta_{i} after K_b; beta_{i-1} during K_a)
    int* active;        // [k]
    int* n_active;      // [1]
    double* part;       // [GX*k]
    unsigned* ticket;   // [4]
    // The Lanczos vectors are stored unnormalised: v_i = scur * U_i (U_i = the orthogonalised
    // residual of the previous step) and v_{i-1} = sprev * U_{i-1}; the products and the
    // orthogonalisation apply the scales on the fly, so no separate normalisation pass runs.
    double* scur;       // [k] 1/beta_{i-1} (0 for stopped columns)
    double* sprev;      // [k] 1/beta_{i-2}
    int maxn, k;
};

int apply_kron(const edx_kron* K, const void* tmap, const double2* Vc, double2* Vp, const KrylovState& S, int it,
               unsigned* tile_ticket, int* err, int col_group, int blocks_per_sm, cudaStream_t st);
int kron_tensor_map(const edx_kron* K, const double2* X, int k, int col_group, void* tmap_out);
int kron_check(const edx_kron* K);
int kron_grid_x(const edx_kron* K, int k, int col_group, int blocks_per_sm);
int kron_col_group(int k, int requested);

}  // namespace edx
