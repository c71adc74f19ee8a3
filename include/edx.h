/*
 * edx.h -- C ABI of libedx, the B200 (sm_100a) exact-diagonalisation core behind the
 * ED/XAS/RIXS solvers of EDRIXS.
 *
 * Plain pointers and sizes only.  Pointers named d_* are device pointers on the current
 * CUDA device; `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 * Every function returns an EDX_* status; on failure edx_last_error() holds a message.
 * Nothing here aborts the process (the reference STOPs instead, src/io.f90:37-39).
 *
 * Layouts
 *   complex128 = two doubles (re, im); complex64 = two floats.
 *   CSR: row_ptr int64[nrows+1] 0-based, col int32[nnz] 0-based and ascending within a
 *   row, val complex128 or complex64[nnz].  The reference's CSR (src/m_types.f90:39-54)
 *   is 1-based int32; subtract one from its iaa/jaa to compare.
 *   Multi-vector blocks X are row-major: element (row r, column c) at X[r*ld + c].
 *
 * Workspace: entry points that need scratch take (d_work, work_bytes) from the caller and
 * report the size they need through the matching *_workspace() query.
 */
#ifndef EDX_H
#define EDX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDX_ABI_VERSION 7

/* status codes */
#define EDX_OK 0
#define EDX_ERR_INVALID 1       /* bad argument */
#define EDX_ERR_CUDA 2          /* a CUDA call failed */
#define EDX_ERR_WORKSPACE 3     /* caller workspace too small */
#define EDX_ERR_ROW_CAPACITY 4  /* a row produced more candidate entries than supported */
#define EDX_ERR_OVERFLOW 5      /* index does not fit the index type */

/* value types */
#define EDX_C128 0
#define EDX_C64 1

/* build modes (src/ham.f90) */
#define EDX_HAM_I 0   /* build_ham_i      src/ham.f90:2-349    */
#define EDX_HAM_N 1   /* build_ham_n      src/ham.f90:352-711  */
#define EDX_TRANS_I 2 /* build_transop_i  src/ham.f90:714-912  */
#define EDX_TRANS_F 3 /* build_transop_f  src/ham.f90:915-1115 */

const char* edx_last_error(void);
int edx_abi_version(void);

/* ---------------------------------------------------------------------------------- */
/* Fock basis                                                                          */
/* ---------------------------------------------------------------------------------- */

/* Number of norb-bit states with nelec electrons, C(norb, nelec); norb <= 63. */
int edx_fock_count(int norb, int nelec, int64_t* ndim);

/* All norb-bit states with popcount nelec in ascending order, by combinatorial unranking.
 * Replaces get_fock_full_N + sort + write/read of fock_*.in
 * (edrixs/fock_basis.py:133-172, :398-451; src/io.f90:174-361). */
int edx_fock_unrank(int norb, int nelec, uint64_t* d_fock, int64_t ndim, void* stream);

/* *is_full = 1 if d_fock[0..ndim) is exactly the full norb/nelec basis (then column lookups
 * may use combinatorial ranking instead of src/utils.f90:2-40 binary search). Synchronises. */
int edx_fock_match_full(int norb, int nelec, const uint64_t* d_fock, int64_t ndim, int* is_full,
                        void* d_work, size_t work_bytes, void* stream);
int edx_fock_match_full_workspace(size_t* bytes);

/* ---------------------------------------------------------------------------------- */
/* Hamiltonian / transition-operator CSR build: two passes (count, then fill) exactly as   */
/* src/ham.f90:59-188 and :213-346: per row, terms in file order (hopping, then Coulomb,  */
/* then the omega diagonal when ham_sign < 0), fermion signs from popcounts, columns      */
/* ascending, duplicates summed in term order, explicit zeros kept                        */
/* (src/m_types.f90:74-121).                                                              */
/* ---------------------------------------------------------------------------------- */
typedef struct edx_build_desc {
    int mode;                      /* EDX_HAM_I / EDX_HAM_N / EDX_TRANS_I / EDX_TRANS_F */
    const uint64_t* fock_left;     /* row-side valence basis (device), ascending */
    int64_t ndim_left;
    const uint64_t* fock_right;    /* column-side valence basis for TRANS_I/TRANS_F */
    int64_t ndim_right;
    int num_val_orbs;              /* nv: core bits sit above the nv valence bits */
    int num_core_orbs;             /* nc */
    int search_norb, search_nelec; /* >0: the searched basis is the full set -> ranking */
    int nhopp;                     /* two-fermion terms (hopping / transop files) */
    const int32_t* hopp_idx;       /* device int32[2*nhopp], 1-based as in the files */
    const double* hopp_val;        /* device complex128[nhopp] */
    int ncoul;                     /* four-fermion terms (HAM modes only) */
    const int32_t* coul_idx;       /* device int32[4*ncoul], 1-based */
    const double* coul_val;        /* device complex128[ncoul] */
    double ham_sign;               /* HAM modes: multiplies every term value */
    double omega_re, omega_im;     /* HAM modes with ham_sign < 0: added on the diagonal */
} edx_build_desc;

int64_t edx_build_nrows(const edx_build_desc* d);
int64_t edx_build_ncols(const edx_build_desc* d);
int edx_build_workspace(const edx_build_desc* d, size_t* bytes);
/* Pass 1: d_row_nnz[nrows] = merged entries per row; *cap_out = the per-row candidate
 * capacity that the fill pass must be given.  Synchronises (reads an overflow flag). */
int edx_build_count(const edx_build_desc* d, int32_t* d_row_nnz, int* cap_out, void* d_work,
                    size_t work_bytes, void* stream);
/* Exclusive scan of the row counts into d_row_ptr[nrows+1]; *h_nnz = total (synchronises). */
int edx_build_scan(const int32_t* d_row_nnz, int64_t nrows, int64_t* d_row_ptr, int64_t* h_nnz,
                   void* d_work, size_t work_bytes, void* stream);
int edx_build_scan_workspace(int64_t nrows, size_t* bytes);
/* Pass 2: columns and values at d_row_ptr[r]; d_val64 (complex64 copy) may be NULL, and
 * d_val may be NULL when d_val64 is given (a complex64-only matrix). */
int edx_build_fill(const edx_build_desc* d, int cap, const int64_t* d_row_ptr, int32_t* d_col,
                   double* d_val, float* d_val64, void* d_work, size_t work_bytes, void* stream);

/* ---------------------------------------------------------------------------------- */
/* Sparse products                                                                     */
/* ---------------------------------------------------------------------------------- */
typedef struct edx_csr {
    int64_t nrows, ncols, nnz;
    const int64_t* row_ptr;
    const int32_t* col;
    const void* val;
    int val_type; /* EDX_C128 or EDX_C64 */
} edx_csr;

/* Y = alpha*(A X) + sigma*X + beta*Y over k columns (sigma needs nrows == ncols).
 * With beta = 1, sigma = 0 this is matvec_csr's y += A x (src/spmv.f90:73-103, the
 * per-rank kernel of pspmv_csr src/spmv.f90:1-71).  vec_type: EDX_C128 or EDX_C64 for X
 * and Y; C64 X/Y require a C64 matrix (complex64 arithmetic).  col_group: columns handled
 * per lane group of a warp (1, 2, 4, 6, 8, 12, 16 or 32; 0 = the smallest of those >= k,
 * capped at 32 with column tiles beyond). */
int edx_spmm(const edx_csr* A, int k, int vec_type, const void* d_x, int64_t ldx, void* d_y,
             int64_t ldy, double alpha_re, double alpha_im, double sigma_re, double sigma_im,
             double beta_re, double beta_im, int col_group, void* stream);

/* ---------------------------------------------------------------------------------- */
/* Packed form of a square matrix (no counterpart in the reference)                    */
/* ---------------------------------------------------------------------------------- */

/* A Hamiltonian built from a few hundred hopping and Coulomb terms has only a few hundred
 * distinct off-diagonal values (for example 423 bit patterns in the 11.0 M off-diagonal
 * entries of a 184,756-state impurity model).  The packed form keeps the diagonal as a
 * dense complex128 vector and stores every off-diagonal entry by its column and an index
 * into vals (the distinct values, bit-exact copies).  Rows keep the CSR's column order.
 * Two forms:
 *   narrow (vbits >= 1): one 32-bit word, ent = column << vbits | index, with
 *     vbits = 32 - (bits of ncols-1); it exists when nval <= min(2^vbits, EDX_PACK_VALUES_MAX);
 *   wide (vbits == 0): ent = column and vidx = index (16 bits), 6 bytes per entry, for
 *     matrices whose column needs too many of the 32 bits (tens of millions of states);
 *     it exists when nval <= EDX_PACK_VALUES_MAX. */
#define EDX_PACK_VALUES_MAX 2048
#define EDX_PACK_AUTO 0    /* narrow when it fits, else wide */
#define EDX_PACK_NARROW 1
#define EDX_PACK_WIDE 2
typedef struct edx_packed {
    int64_t nrows;
    int64_t nnz;               /* off-diagonal entries */
    const int64_t* row_ptr;    /* device int64[nrows+1] */
    const uint32_t* ent;       /* device uint32[nnz] */
    int vbits;                 /* 0: wide form */
    int nval;
    const double* vals;        /* device complex128[nval] */
    const double* diag;        /* device complex128[nrows]; zero where the CSR has no diagonal */
    const uint16_t* vidx;      /* wide form: device uint16[nnz]; NULL for the narrow form */
} edx_packed;

/* The count pass sorts the off-diagonal values in chunks of at most 2^26 entries, so the
 * workspace stays near 40 bytes x min(nnz, 2^26) + 32 bytes x nrows at any size. */
int edx_pack_workspace(const edx_csr* A, size_t* bytes);
/* Pass 1: *nnz_off, *nval, *vbits (0 = wide) of complex128 square A, in the requested form
 * (EDX_PACK_AUTO / _NARROW / _WIDE).  EDX_ERR_OVERFLOW when A has too many distinct
 * off-diagonal values for that form.  Synchronises `stream`. */
int edx_pack_count(const edx_csr* A, int form, int64_t* nnz_off, int* nval, int* vbits, void* d_work,
                   size_t work_bytes, void* stream);
/* Pass 2: P->nnz, nval, vbits from pass 1 and its arrays (vidx too for the wide form)
 * allocated by the caller; d_work must still hold what pass 1 left in it. */
int edx_pack_fill(const edx_csr* A, edx_packed* P, void* d_work, size_t work_bytes, void* stream);
/* edx_spmm on the packed form: Y = alpha*(A X) + sigma*X + beta*Y over k complex128 columns
 * (matvec_csr, src/spmv.f90:73-103, on the packed matrix).  The distinct values sit in
 * shared memory; the diagonal term is added per row.  col_group as for edx_spmm. */
int edx_spmm_packed(const edx_packed* P, int k, const double* d_x, int64_t ldx, double* d_y, int64_t ldy,
                    double alpha_re, double alpha_im, double sigma_re, double sigma_im, double beta_re,
                    double beta_im, int col_group, void* stream);

/* ---------------------------------------------------------------------------------- */
/* Slab form of an impurity-model Hamiltonian (no counterpart in the reference, whose     */
/* matvec_csr src/spmv.f90:73-103 walks a flat CSR built by src/ham.f90:2-711)          */
/* ---------------------------------------------------------------------------------- */

/* When the two-body terms touch only the "A" orbitals (impurity and core) and the bath
 * orbitals carry only their levels and the A-bath hybridisation, every Fock state is a pair
 * (I, B) of an A configuration and a bath configuration, and
 *   H = H_A (x) 1 + diag(d_B) + sum_{a,b} t_cre[a][b] c+_a c_b + t_ann[a][b] c+_b c_a.
 * Rows are grouped by I into slabs (slab s = rows slab_off[s] .. slab_off[s+1]-1, its bath
 * configurations in colex order of sector slab_m[s]), so the product reads whole source
 * slabs: those of H_A's row s, and the slabs I +- a one bath electron away.  Rows here are in
 * slab order; the host keeps the permutation to the reference's row order.  Built on the host
 * (edrixs_b200/kron.py) from the term lists; bath tables index b_off[m] + rank.  Signs:
 * A-side factors come from the compressed A configuration slab_cfg[s] (A orbitals numbered
 * by ascending full-state bit, the n_alo below the bath first), bath-side factors from the
 * bath configuration; the formulas are in edrixs_b200/kron.py. */
#define EDX_KRON_NB_MAX 16
#define EDX_KRON_NAH_MAX 16
/* source kinds of slab s (src_kind = kind | q << 4) */
#define EDX_KRON_SRC_HA 0    /* another slab of H_A's row s: Y += coef X_src */
#define EDX_KRON_SRC_OWN 1   /* slab s itself: Y += (coef + b_diag[B]) X_s (coef = H_A's diagonal) */
#define EDX_KRON_SRC_CRE 2   /* slab I + a_q: Y(B) += sum_{b in B} sign t_cre[q][b] X_src(B - b) */
#define EDX_KRON_SRC_ANN 3   /* slab I - a_q: Y(B) += sum_{b not in B} sign t_ann[q][b] X_src(B + b) */
typedef struct edx_kron {
    int64_t nrows;
    int32_t nslab, nb, nah, n_alo;
    int32_t max_rows;           /* rows of the largest slab */
    const int32_t* slab_off;    /* device int32[nslab+1] */
    const int32_t* slab_m;      /* device int32[nslab] bath electrons */
    const uint32_t* slab_cfg;   /* device uint32[nslab] compressed A configuration */
    const int32_t* hyb_a;       /* device int32[nah]: compressed A index a_q */
    const double* t_cre;        /* device complex128[nah*nb]: coefficient of c+_{a_q} c_b */
    const double* t_ann;        /* device complex128[nah*nb]: coefficient of c+_b c_{a_q} */
    const int64_t* src_ptr;     /* device int64[nslab+1]: sources of slab s, own slab first */
    const int32_t* src_slab;    /* device int32[nsrc] */
    const int32_t* src_kind;    /* device int32[nsrc] */
    const double* src_coef;     /* device complex128[nsrc] (H_A entries; 0 for CRE / ANN) */
    const int32_t* b_off;       /* device int32[nb+2] */
    const uint16_t* b_cfg;      /* device uint16[2^nb] */
    const uint16_t* b_nbr;      /* device uint16[2^nb * nb]: rank of cfg ^ (1 << x) in its sector */
    const double* b_diag;       /* device complex128[2^nb] */
} edx_kron;

/* Variants of the slab product (the col_group argument of edx_kron_spmm, apply_col_group of
 * edx_krylov_opts with apply_kron; other values mean EDX_KRON_AUTO).  STAGED: the source
 * slabs are staged in shared memory by the tensor-memory accelerator (2-D tiled loads of
 * 32-row boxes; no multicast); it needs slabs of at most 1024 rows whose ring of three
 * staged slabs fits in shared memory (about 590 rows: up to 11 bath orbitals).  GATHER: every
 * thread reads its row's source rows from global memory (any slab size).  AUTO: GATHER for
 * up to 8 columns or when STAGED does not fit, else STAGED (the faster of the two on wide
 * blocks). */
#define EDX_KRON_AUTO 0
#define EDX_KRON_STAGED 1
#define EDX_KRON_GATHER 2
/* Y = H X in slab order for k columns (row-major, ld = k), on the slab form, in the variant
 * col_group selects (above).  EDX_ERR_CUDA if a staged load did not arrive within its time
 * limit; EDX_ERR_INVALID if a slab or a source row lies outside the descriptor's ranges (the
 * kernels record both in the workspace and skip the access).  X and Y must not overlap. */
int edx_kron_spmm_workspace(size_t* bytes);
int edx_kron_spmm(const edx_kron* K, int k, const double* d_x, double* d_y, int col_group, void* d_work,
                  size_t work_bytes, void* stream);

/* dst[i*ld_dst + c] = src[idx[i]*ld_src + c] for i < n, c < k (complex128): moves blocks
 * between the reference's row order and the slab order (idx = the permutation, or its
 * inverse). */
int edx_permute_rows(int64_t n, int k, const double* d_src, int64_t ld_src, const int64_t* d_idx, double* d_dst,
                     int64_t ld_dst, void* stream);

/* ---------------------------------------------------------------------------------- */
/* Block Gram-Schmidt for the ground-state eigensolver (the reorthogonalisation inside      */
/* ARPACK's pznaupd, src/arpack.f90:76, done here for the thick-restart Lanczos)          */
/* ---------------------------------------------------------------------------------- */

/* V: m basis vectors of length n, vector i at d_V[i*ldv .. i*ldv + n) (complex128).
 * W: n x k block, row-major (d_W[r*k + c]), 1 <= k <= 8.  C: m x k row-major.
 * edx_gs_dot:    C = V^H W   (deterministic: fixed row chunks per block, fixed final tree)
 * edx_gs_update: W -= V^T C
 * (m + 512) * k * 16 bytes must fit in 200 KB. */
int edx_gs_workspace(int m, int k, size_t* bytes);
int edx_gs_dot(const double* d_V, int m, int64_t n, int64_t ldv, const double* d_W, int k, double* d_C,
               void* d_work, size_t work_bytes, void* stream);
int edx_gs_update(const double* d_V, int m, int64_t n, int64_t ldv, double* d_W, int k, const double* d_C,
                  void* stream);
/* The two passes of CholeskyQR for the block W (n x k row-major, k <= 8):
 * edx_gs_gram: G = W^H W (k x k row-major; deterministic as edx_gs_dot; workspace from
 *              edx_gs_workspace(k, k, ...))
 * edx_gs_rmul: W = W M for a k x k row-major M (e.g. the inverse Cholesky factor). */
int edx_gs_gram(const double* d_W, int64_t n, int k, double* d_G, void* d_work, size_t work_bytes, void* stream);
int edx_gs_rmul(double* d_W, int64_t n, int k, const double* d_M, void* stream);

/* ---------------------------------------------------------------------------------- */
/* Lanczos / Krylov                                                                     */
/* ---------------------------------------------------------------------------------- */

/* Optional extras of edx_krylov (pass NULL for none).
 *
 * Projections: every normalised Lanczos vector v_i (i = 0..maxn-1, v_0 = v0/|v0|) of every
 *   column j is multiplied by each CSR proj[p] (e.g. an emission operator) and stored
 *   column-major per column: proj_out[p][(j*maxn + i)*proj[p].nrows + r].
 * Shifted solves: for each shift s (column shift_col[s], complex shift_z[s]) the MINRES
 *   recurrence of pminres_csr (src/linsys.f90:3-128) for (z - A) x = v0_j is carried in the
 *   Lanczos basis of A: the Lanczos vectors of z - A are +-those of A and its alpha is
 *   z - alpha, so all shifts of one column share one Krylov space.  Each shift stops on its
 *   own with the reference's rule (|res| <= shift_tol or iterations >= shift_maxit) and the
 *   loop ends when every shift has stopped.  Output: x_s = sum_i shift_y[s*maxn + i] v_i
 *   (complex128 coefficients), shift_iters[s], shift_res[s]. */
typedef struct edx_krylov_opts {
    int nproj;
    const edx_csr* proj;         /* host array of nproj matrices */
    double* const* proj_out;     /* host array of nproj device pointers */
    int nshift;
    const int32_t* shift_col;    /* device int32[nshift] */
    const double* shift_z;       /* device complex128[nshift] */
    double shift_tol;
    int shift_maxit;
    double* shift_y;             /* device complex128[nshift*maxn] */
    int32_t* shift_iters;        /* device int32[nshift] */
    double* shift_res;           /* device double[nshift] */
    /* optional instrumentation (host pointers, may be NULL): total device time of the fused
     * SpMM + recurrence launches (the dominant kernel), measured with CUDA events recorded
     * on `stream` around each launch, and the number of those launches */
    double* apply_ms;
    int* apply_launches;
    /* launch shape of the fused SpMM + recurrence kernel (0 = default): columns per lane
     * group (1, 2, 4, 6, 8, 12, 16 or 32), threads per block (256 or 1024), blocks per SM,
     * row mapping (0 = interleaved rows, 1 = one contiguous row range per block), and
     * column tiles per block (1, 2 or 4; group widths 16 and 32 only), and whether each
     * warp bulk-prefetches its next row into L2 (cp.async.bulk.prefetch) */
    int apply_col_group;
    int apply_threads;
    int apply_blocks_per_sm;
    int apply_chunked;
    int apply_tiles;
    int apply_prefetch;
    /* packed form of the same matrix (edx_pack_fill), or NULL.  With it the product reads
     * one 32-bit word per off-diagonal entry and the value from a table in shared memory,
     * with the launch-shape fields above. */
    const edx_packed* apply_packed;
    /* slab form of the same matrix, or NULL.  With it the product is k_lanczos_apply_kron
     * (or k_lanczos_apply_kron_gather: apply_col_group selects the EDX_KRON_* variant):
     * the start vectors d_v0 and every Lanczos vector are in slab order, and A is used for
     * its shape only.  Projections need operators whose columns are in slab order too. */
    const edx_kron* apply_kron;
    /* streaming projections, for problems where P_p V (every projected Lanczos vector) does
     * not fit in memory.  With proj_window = B > 0, proj_out[p] holds only the last B
     * projected vectors (device complex128[k][B][nrows_p]) and every B iterations (and at
     * the end) they are folded into nacc accumulators:
     *   acc_out[p][r * acc_ld + s] += sum_i acc_coef[s * maxn + i] * (P_p v_i)[column acc_col[s]][r]
     * so that P_p (V y_s) is formed for coefficient vectors y_s (for example the per-shift
     * MINRES coefficients of an earlier call with the same start vectors). */
    int proj_window;
    int nacc;
    const int32_t* acc_col;      /* device int32[nacc]: Lanczos column of accumulator s */
    const double* acc_coef;      /* device complex128[nacc * maxn] */
    double* const* acc_out;      /* host array of nproj device pointers */
    int64_t acc_ld;
    /* leading dimension of d_v0 (0 = k): the start vectors may be k columns of a wider
     * row-major block */
    int64_t v0_ld;
    /* with k <= apply_col_group <= 16 (CSR or packed form): each lane group walks a row of
     * its own (no reduction across the groups of a warp per row) */
    int apply_rowslot;
} edx_krylov_opts;

/* k independent Lanczos recurrences of build_krylov_mp (src/lanczos.f90:210-303), run
 * together so that every iteration is one SpMM over k columns (FP64 recurrence).  d_v0:
 * n x k start vectors, row-major with leading dimension opts->v0_ld (k when 0).  Outputs
 * for column j: d_alpha[j*maxn + i], d_beta[j*maxn + i] (i < neff), d_norm[j] =
 * <v0_j|v0_j>, d_neff[j].  Column j stops when beta < 1e-10 (absolute, :291); a zero start
 * vector gives neff = 1 and norm 0.  The matrix may be complex128 or complex64 (vectors and
 * scalars stay complex128 / FP64). */
int edx_krylov_workspace(int64_t n, int k, const edx_krylov_opts* opts, int maxn, size_t* bytes);
int edx_krylov(const edx_csr* A, int k, const double* d_v0, int maxn, double* d_alpha,
               double* d_beta, double* d_norm, int32_t* d_neff, const edx_krylov_opts* opts,
               void* d_work, size_t work_bytes, void* stream);

/* MINRES of pminres_csr (src/linsys.f90:3-128) for one right-hand side, x0 = 0, with the
 * same complex Givens recurrences and stopping rule (|res| <= tol or iter >= maxit).
 * A is applied as alpha*(A x) + sigma*x (alpha = 1, sigma = 0 reproduces the reference,
 * which stores omega + E_g + i*gamma - H_n explicitly; alpha = -1, sigma = z applies the
 * same operator to a resident H_n without rebuilding it). */
int edx_minres_workspace(int64_t n, size_t* bytes);
int edx_minres(const edx_csr* A, double alpha_re, double alpha_im, double sigma_re,
               double sigma_im, const double* d_b, double* d_x, double tol, int maxit,
               int* iters_out, double* res_out, void* d_work, size_t work_bytes, void* stream);

/* Final-state start vectors of the batched RIXS from stored projections (the D_out^+ x of
 * src/rixs_driver.f90 for every shift, after edx_krylov with stored proj_out):
 *   d_out[r*ld_out + (p*k + c)*nw + w] = sum_{i<m} y[(c*nw + w)*ldy + i] * proj_p[(c*maxn + i)*nrows + r]
 * for p < np, c < k, w < nw, r < nrows (complex128): proj_p = d_proj[p] (host array of np
 * device pointers, the [k][maxn][nrows] blocks edx_krylov writes), y the shifts' MINRES
 * coefficients in the Lanczos basis (shift_y: column c's nw shifts, rows of length ldy >= m),
 * m <= maxn the Lanczos vectors used.  Each output is one sum over i in order. */
int edx_proj_combine(int np, const double* const* d_proj, int k, int maxn, int m, int64_t nrows,
                     const double* d_y, int64_t ldy, int nw, double* d_out, int64_t ld_out, void* stream);

/* Continued fraction of get_spectra_from_poles (edrixs/plot_spectrum.py:41-61) for nset
 * pole sets on one grid:  spec[w] (+)= sum_s weight[s] * norm[s] * (-1/pi) *
 * Im 1/(x - a_1 - b_1^2/(x - a_2 - ...)),  x = omega[w] + i*gamma[w] + e0[s].
 * Pole set s: neff[s] coefficients at d_alpha[s*ld], d_beta[s*ld].  With per_set != 0 the
 * output is d_spec[s*ngrid + w] (no sum over s). */
int edx_cf_spectrum(int nset, const int32_t* d_neff, const double* d_alpha, const double* d_beta,
                    int ld, const double* d_e0, const double* d_norm, const double* d_weight,
                    int ngrid, const double* d_omega, const double* d_gamma, double* d_spec,
                    int per_set, int accumulate, void* stream);

/* Density matrix of ed_driver.f90:194-248 for nvec eigenvectors (n x nvec, ld = nvec) over
 * the ascending basis d_fock: d_out[(v*nv + i)*nv + j] = the reference's denmat(i+1, j+1, v+1)
 * (complex128).  Off-diagonal terms skip rows whose amplitude is below 1e-10 as the
 * reference does.  Deterministic (row chunks summed in order). */
int edx_denmat_workspace(int64_t n, int nv, int nvec, size_t* bytes);
int edx_denmat(const uint64_t* d_fock, int64_t n, int search_norb, int search_nelec, int nv,
               int nvec, const double* d_vecs, double* d_out, void* d_work, size_t work_bytes,
               void* stream);

/* The density matrix of edx_denmat for callers that cannot allocate device memory and so
 * cannot pass a workspace (no counterpart in the reference, which allocates as it pleases).
 * Examples: a host whose HBM is carved up in advance by its own allocator, or a thin
 * foreign-language binding that only forwards buffers it was handed.  The partial sums live
 * in a fixed file-scope device array of EDX_DENMAT_STATIC_CHUNKS x
 * EDX_DENMAT_STATIC_MAX_ENTRIES complex128 values (4 MiB) that every GPU loading the library
 * holds until the process exits.  Limit: nvec * nv * nv <= EDX_DENMAT_STATIC_MAX_ENTRIES,
 * otherwise EDX_ERR_INVALID.  Every call looks up the array's device address
 * (cudaGetSymbolAddress) with the calling device current, so the address stays right after
 * a cudaDeviceReset; the first call on a device may load the library's device code, so make
 * it before any stream capture.  All calls share the one array: calls that overlap on the GPU
 * (for example on two streams) race and must be serialised by the caller.  Allocates nothing. */
#define EDX_DENMAT_STATIC_CHUNKS 64
#define EDX_DENMAT_STATIC_MAX_ENTRIES 4096
#define EDX_MAX_DEVICES 64
int edx_denmat_static(const uint64_t* d_fock, int64_t n, int search_norb, int search_nelec,
                      int nv, int nvec, const double* d_vecs, double* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EDX_H */
