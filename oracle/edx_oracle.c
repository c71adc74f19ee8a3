/*
 * edx_oracle.c -- CPU FP64 restatement of the EDRIXS Fortran hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is compiled into
 * oracle/libedx_oracle.so and loaded by tests/, by __graft_entry__.smoke() to check its
 * results, and by bench.py's CPU-baseline leg.  The product path (edrixs_b200) never
 * links or calls it.
 *
 * Every routine restates one reference routine (paths relative to the reference repo):
 *   orc_fock_full_N      edrixs/fock_basis.py:133-172 (+ the sort at :444)
 *   orc_binary_search    src/utils.f90:2-40
 *   orc_make_newfock     src/fock.f90:38-68
 *   orc_build_count/fill src/ham.f90:2-349   build_ham_i      (mode 0)
 *                        src/ham.f90:352-711 build_ham_n      (mode 1)
 *                        src/ham.f90:714-912 build_transop_i  (mode 2)
 *                        src/ham.f90:915-1115 build_transop_f (mode 3)
 *                        with the sorted-insert-with-merge row list of
 *                        src/m_types.f90:74-121 (columns ascending, equal columns summed
 *                        in term order, zeros kept)
 *   orc_matvec           src/spmv.f90:73-103 (y += A x, row sums in CSR order)
 *   orc_build_krylov     src/lanczos.f90:210-303
 *   orc_minres           src/linsys.f90:3-128
 *   orc_denmat           src/ed_driver.f90:194-248
 *
 * Index conventions: the reference stores 1-based rows/columns; this oracle returns
 * 0-based row pointers (int64) and 0-based column indices (int32).  Complex numbers are
 * interleaved (re, im) doubles.  Parity against the reference's own Python builder and its
 * known-answer test is checked in tests/test_oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------------------ */
/* Fock basis                                                                           */
/* ------------------------------------------------------------------------------------ */

int64_t orc_binomial(int n, int k) {
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    unsigned __int128 r = 1;
    for (int i = 1; i <= k; ++i) r = r * (unsigned)(n - k + i) / (unsigned)i;
    return (int64_t)r;
}

/* All norb-bit integers with popcount N, ascending (fock_basis.py:133-172 builds them from
 * half-shell blocks; write_fock_dec_by_N sorts them at :444).  Here: Gosper's hack walks
 * the same set directly in ascending order. */
int64_t orc_fock_full_N(int norb, int N, int64_t *out) {
    if (norb < 0 || norb > 62 || N < 0 || N > norb) return -1;
    int64_t n = orc_binomial(norb, N);
    if (!out) return n;
    if (N == 0) { out[0] = 0; return 1; }
    uint64_t v = (N == 64) ? ~0ull : ((1ull << N) - 1ull);
    for (int64_t i = 0; i < n; ++i) {
        out[i] = (int64_t)v;
        uint64_t t = v | (v - 1);
        v = (t + 1) | (((~t & -~t) - 1) >> (__builtin_ctzll(v) + 1));
    }
    return n;
}

/* utils.f90:2-40: 1-based position of m in ascending vec(1:n), -1 if absent. */
int64_t orc_binary_search(int64_t n, const int64_t *vec, int64_t m) {
    int64_t left = 1, right = n;
    while (left <= right) {
        int64_t middle = left + (right - left) / 2;
        if (vec[middle - 1] < m) left = middle + 1;
        else if (vec[middle - 1] > m) right = middle - 1;
        else return middle;
    }
    return -1;
}

/* fock.f90:38-68: sign = (-1)^(number of occupied orbitals below pos); pos is 1-based.
 * '+' adds 2^(pos-1), '-' subtracts it (callers have already tested the bit). */
void orc_make_newfock(char c_type, int pos, int64_t old, int64_t *new_, int *sgn) {
    int cnt = 0;
    for (int i = 1; i <= pos - 1; ++i)
        if ((old >> (i - 1)) & 1) cnt++;
    *sgn = (cnt % 2) ? -1 : 1;
    if (c_type == '+') *new_ = old + ((int64_t)1 << (pos - 1));
    else *new_ = old - ((int64_t)1 << (pos - 1));
}

static inline int btest(int64_t x, int pos0) { return pos0 >= 0 && pos0 < 63 && ((x >> pos0) & 1); }

/* ------------------------------------------------------------------------------------ */
/* CSR build (ham.f90)                                                                   */
/* ------------------------------------------------------------------------------------ */

typedef struct {
    int mode;                 /* 0 ham_i, 1 ham_n, 2 transop_i, 3 transop_f */
    const int64_t *fock_left; /* row-side valence basis */
    int64_t ndim_left;
    const int64_t *fock_right;/* column-side valence basis (modes 2, 3); ignored otherwise */
    int64_t ndim_right;
    int num_val_orbs;
    int num_core_orbs;
    int nhopp;                /* two-fermion terms: idx[2*t], idx[2*t+1] (1-based), val re/im */
    const int32_t *hopp_idx;
    const double *hopp_val;
    int ncoul;                /* four-fermion terms: idx[4*t..4*t+3] (1-based) */
    const int32_t *coul_idx;
    const double *coul_val;
    double ham_sign;
    double omega_re, omega_im;
} orc_build_t;

int64_t orc_build_nrows(const orc_build_t *b) {
    switch (b->mode) {
    case 0: return b->ndim_left;
    case 1: return b->ndim_left * b->num_core_orbs;
    case 2: return b->ndim_left * b->num_core_orbs;
    case 3: return b->ndim_left;
    }
    return -1;
}

typedef struct { int32_t col; double re, im; } orc_entry;

/* sorted insert with merge: m_types.f90:74-121 (init_col / insert_into_row) */
static void row_insert(orc_entry *row, int *n, int32_t col, double re, double im) {
    int i = 0;
    while (i < *n && row[i].col < col) i++;
    if (i < *n && row[i].col == col) { row[i].re += re; row[i].im += im; return; }
    memmove(row + i + 1, row + i, sizeof(orc_entry) * (size_t)(*n - i));
    row[i].col = col; row[i].re = re; row[i].im = im;
    (*n)++;
}

/* Row state and column lookup per mode (ham.f90:59-176 / :414-446 / :772-800 / :970-990). */
static int64_t row_state(const orc_build_t *b, int64_t icfg /*1-based*/, const int64_t *fock_core) {
    int nv = b->num_val_orbs, nc = b->num_core_orbs;
    if (b->mode == 0) return b->fock_left[icfg - 1];
    if (b->mode == 3) return (((int64_t)1 << nc) - 1) * ((int64_t)1 << nv) + b->fock_left[icfg - 1];
    int64_t core_indx = (icfg - 1) / b->ndim_left + 1;
    int64_t val_indx = (icfg - 1) % b->ndim_left + 1;
    return fock_core[core_indx - 1] * ((int64_t)1 << nv) + b->fock_left[val_indx - 1];
}

/* returns 1-based column or -1 */
static int64_t col_lookup(const orc_build_t *b, int64_t new_, const int64_t *fock_core) {
    int nv = b->num_val_orbs, nc = b->num_core_orbs;
    if (b->mode == 0) return orc_binary_search(b->ndim_left, b->fock_left, new_);
    int64_t p = (int64_t)1 << nv;
    int64_t new_core = new_ / p;
    int64_t new_val = new_ - new_core * p;
    if (b->mode == 2) return orc_binary_search(b->ndim_right, b->fock_right, new_val);
    const int64_t *fr = (b->mode == 1) ? b->fock_left : b->fock_right;
    int64_t nr = (b->mode == 1) ? b->ndim_left : b->ndim_right;
    int64_t kcfg = orc_binary_search(nc, fock_core, new_core);
    int64_t lcfg = orc_binary_search(nr, fr, new_val);
    if (kcfg == -1 || lcfg == -1) return -1;
    return (kcfg - 1) * nr + lcfg;
}

/* Build one row's sorted, merged entry list in reference term order. */
static int build_row(const orc_build_t *b, int64_t icfg, const int64_t *fock_core,
                     orc_entry *row) {
    int n = 0;
    int64_t s0 = row_state(b, icfg, fock_core);
    int is_ham = (b->mode == 0 || b->mode == 1);
    double hs = is_ham ? b->ham_sign : 1.0;
    for (int t = 0; t < b->nhopp; ++t) {
        int alpha = b->hopp_idx[2 * t], beta = b->hopp_idx[2 * t + 1];
        if (!btest(s0, alpha - 1)) continue;
        int64_t old = s0, nw; int sgn, tot = 1;
        orc_make_newfock('-', alpha, old, &nw, &sgn); tot *= sgn; old = nw;
        if (btest(old, beta - 1)) continue;
        orc_make_newfock('+', beta, old, &nw, &sgn); tot *= sgn;
        int64_t j = col_lookup(b, nw, fock_core);
        if (j == -1) continue;
        /* val * tot_sign * ham_sign: exact sign flips of both components */
        row_insert(row, &n, (int32_t)(j - 1), b->hopp_val[2 * t] * tot * hs,
                   b->hopp_val[2 * t + 1] * tot * hs);
    }
    if (is_ham) {
        for (int t = 0; t < b->ncoul; ++t) {
            const int32_t *ix = b->coul_idx + 4 * t;
            int64_t old = s0, nw; int sgn, tot = 1;
            if (!btest(old, ix[0] - 1)) continue;
            orc_make_newfock('-', ix[0], old, &nw, &sgn); tot *= sgn; old = nw;
            if (!btest(old, ix[1] - 1)) continue;
            orc_make_newfock('-', ix[1], old, &nw, &sgn); tot *= sgn; old = nw;
            if (btest(old, ix[2] - 1)) continue;
            orc_make_newfock('+', ix[2], old, &nw, &sgn); tot *= sgn; old = nw;
            if (btest(old, ix[3] - 1)) continue;
            orc_make_newfock('+', ix[3], old, &nw, &sgn); tot *= sgn;
            int64_t j = col_lookup(b, nw, fock_core);
            if (j == -1) continue;
            row_insert(row, &n, (int32_t)(j - 1), b->coul_val[2 * t] * tot * hs,
                       b->coul_val[2 * t + 1] * tot * hs);
        }
        if (b->ham_sign < 0) row_insert(row, &n, (int32_t)(icfg - 1), b->omega_re, b->omega_im);
    }
    return n;
}

static void make_fock_core(int nc, int64_t *fc) {
    /* ham.f90:419-421: fock_core(i) = 2^nc - 1 - 2^(nc-i) */
    for (int i = 1; i <= nc; ++i) fc[i - 1] = ((int64_t)1 << nc) - 1 - ((int64_t)1 << (nc - i));
}

static int row_cap(const orc_build_t *b) { return b->nhopp + b->ncoul + 2; }

/* Pass 1 (ham.f90:59-188): number of merged entries per row. Returns total nnz. */
int64_t orc_build_count(const orc_build_t *b, int64_t *row_nnz) {
    int64_t nrows = orc_build_nrows(b);
    int64_t fc[64];
    make_fock_core(b->num_core_orbs, fc);
    int64_t total = 0;
#pragma omp parallel reduction(+ : total)
    {
        orc_entry *row = (orc_entry *)malloc(sizeof(orc_entry) * (size_t)row_cap(b));
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < nrows; ++r) {
            int n = build_row(b, r + 1, fc, row);
            row_nnz[r] = n;
            total += n;
        }
        free(row);
    }
    return total;
}

/* Pass 2 (ham.f90:213-346): write merged entries at row_ptr[r]. */
int orc_build_fill(const orc_build_t *b, const int64_t *row_ptr, int32_t *col, double *val) {
    int64_t nrows = orc_build_nrows(b);
    int64_t fc[64];
    make_fock_core(b->num_core_orbs, fc);
#pragma omp parallel
    {
        orc_entry *row = (orc_entry *)malloc(sizeof(orc_entry) * (size_t)row_cap(b));
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < nrows; ++r) {
            int n = build_row(b, r + 1, fc, row);
            int64_t p = row_ptr[r];
            for (int i = 0; i < n; ++i) {
                col[p + i] = row[i].col;
                val[2 * (p + i)] = row[i].re;
                val[2 * (p + i) + 1] = row[i].im;
            }
        }
        free(row);
    }
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* SpMV and the Krylov solvers                                                          */
/* ------------------------------------------------------------------------------------ */

/* spmv.f90:73-103: y(i) += sum_j a(i,j) x(j), inner sum accumulated in CSR order. */
void orc_matvec(int64_t m, const int64_t *row_ptr, const int32_t *col, const double *val,
                const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        int64_t b0 = row_ptr[i], b1 = row_ptr[i + 1];
        if (b0 >= b1) continue;
        double tr = 0, ti = 0;
        for (int64_t j = b0; j < b1; ++j) {
            double ar = val[2 * j], ai = val[2 * j + 1];
            double xr = x[2 * col[j]], xi = x[2 * col[j] + 1];
            tr += ar * xr - ai * xi;
            ti += ar * xi + ai * xr;
        }
        y[2 * i] += tr;
        y[2 * i + 1] += ti;
    }
}

static double zdotc_re(int64_t n, const double *a, const double *b) {
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; ++i) s += a[2 * i] * b[2 * i] + a[2 * i + 1] * b[2 * i + 1];
    return s;
}

static void zdotc(int64_t n, const double *a, const double *b, double *re, double *im) {
    double sr = 0, si = 0;
#pragma omp parallel for reduction(+ : sr, si) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        sr += a[2 * i] * b[2 * i] + a[2 * i + 1] * b[2 * i + 1];
        si += a[2 * i] * b[2 * i + 1] - a[2 * i + 1] * b[2 * i];
    }
    *re = sr;
    *im = si;
}

/* lanczos.f90:210-303 build_krylov_mp.  alpha[maxn], beta[maxn] (beta(1..neff)), *norm =
 * <phi|phi>; returns neff.  Stops when beta_i < 1e-10 (absolute, :291). */
int orc_build_krylov(int64_t n, const int64_t *row_ptr, const int32_t *col, const double *val,
                     const double *init, int maxn, double *alpha, double *beta, double *norm) {
    double *v = (double *)calloc((size_t)(4 * n), sizeof(double));
    double *cur = v, *prev = v + 2 * n;
    memcpy(cur, init, sizeof(double) * 2 * (size_t)n);
    double nrm2 = zdotc_re(n, cur, cur);
    *norm = nrm2;
    double s = sqrt(nrm2);
    for (int64_t i = 0; i < 2 * n; ++i) cur[i] /= s;
    double beta_prev = 0.0;
    int neff = 0;
    for (int it = 0; it < maxn; ++it) {
        alpha[it] = 0; beta[it] = 0;
    }
    for (int it = 1; it <= maxn; ++it) {
        neff = it;
        for (int64_t i = 0; i < 2 * n; ++i) prev[i] = -beta_prev * prev[i];
        orc_matvec(n, row_ptr, col, val, cur, prev);
        double a = zdotc_re(n, cur, prev);
        alpha[it - 1] = a;
        for (int64_t i = 0; i < 2 * n; ++i) prev[i] -= a * cur[i];
        double b = sqrt(zdotc_re(n, prev, prev));
        beta[it - 1] = b;
        if (fabs(b) < 1e-10) break;
        for (int64_t i = 0; i < 2 * n; ++i) prev[i] /= b;
        double *t = cur; cur = prev; prev = t;
        beta_prev = b;
    }
    free(v);
    return neff;
}

/* complex helpers (Smith's algorithm for division, principal sqrt by the half-angle
 * formula); plain C99 complex is avoided so the arithmetic order is explicit. */
typedef struct { double r, i; } zc;
static inline zc zmul(zc a, zc b) { zc c = {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; return c; }
static inline zc zadd(zc a, zc b) { zc c = {a.r + b.r, a.i + b.i}; return c; }
static inline zc zsub(zc a, zc b) { zc c = {a.r - b.r, a.i - b.i}; return c; }
static inline zc zscale(zc a, double s) { zc c = {a.r * s, a.i * s}; return c; }
static inline zc zdiv(zc a, zc b) {
    zc c;
    if (fabs(b.r) >= fabs(b.i)) {
        double t = b.i / b.r, d = b.r + b.i * t;
        c.r = (a.r + a.i * t) / d; c.i = (a.i - a.r * t) / d;
    } else {
        double t = b.r / b.i, d = b.r * t + b.i;
        c.r = (a.r * t + a.i) / d; c.i = (a.i * t - a.r) / d;
    }
    return c;
}
static inline double zabs(zc a) { return hypot(a.r, a.i); }
static inline zc zsqrt(zc a) {
    double m = zabs(a);
    zc c;
    if (m == 0) { c.r = 0; c.i = 0; return c; }
    if (a.r >= 0) { c.r = sqrt(0.5 * (m + a.r)); c.i = a.i / (2 * c.r); }
    else { c.i = copysign(sqrt(0.5 * (m - a.r)), a.i); c.r = a.i / (2 * c.i); }
    return c;
}

/* linsys.f90:3-128 pminres_csr: solves A x = b with x0 = 0 and the reference's complex
 * Givens recurrences.  Returns the iteration count; *res_out = final |res| estimate. */
int orc_minres(int64_t n, const int64_t *row_ptr, const int32_t *col, const double *val,
               const double *b, double *x, double tol, int maxit, double *res_out) {
    double *v = (double *)calloc((size_t)(4 * n), sizeof(double));
    double *w = (double *)calloc((size_t)(4 * n), sizeof(double));
    double *tmp = (double *)calloc((size_t)(2 * n), sizeof(double));
    double *vc = v, *vp = v + 2 * n, *wc = w, *wp = w + 2 * n;
    memset(x, 0, sizeof(double) * 2 * (size_t)n);
    zc sigma0 = {0, 0}, sigma1 = {0, 0}, gamma0 = {1, 0}, gamma1 = {1, 0};
    memcpy(vc, b, sizeof(double) * 2 * (size_t)n);
    double beta0 = sqrt(zdotc_re(n, vc, vc)), beta1;
    zc eta = {beta0, 0}, res = {beta0, 0};
    int iter = 0;
    while (zabs(res) > tol && iter < maxit) {
        iter++;
        for (int64_t i = 0; i < 2 * n; ++i) vc[i] /= beta0;
        memset(tmp, 0, sizeof(double) * 2 * (size_t)n);
        orc_matvec(n, row_ptr, col, val, vc, tmp);
        zc alpha;
        zdotc(n, vc, tmp, &alpha.r, &alpha.i);
        for (int64_t i = 0; i < n; ++i) {
            zc t = {tmp[2 * i], tmp[2 * i + 1]}, c = {vc[2 * i], vc[2 * i + 1]};
            zc p = {vp[2 * i], vp[2 * i + 1]};
            zc r = zsub(zsub(t, zmul(alpha, c)), zscale(p, beta0));
            vp[2 * i] = r.r; vp[2 * i + 1] = r.i;
        }
        beta1 = sqrt(zdotc_re(n, vp, vp));
        zc delta = zsub(zmul(gamma0, alpha), zscale(zmul(gamma1, sigma0), beta0));
        zc b1 = {beta1, 0};
        zc rho1 = zsqrt(zadd(zmul(delta, delta), zmul(b1, b1)));
        zc rho2 = zadd(zmul(sigma0, alpha), zscale(zmul(gamma1, gamma0), beta0));
        zc rho3 = zscale(sigma1, beta0);
        gamma1 = gamma0;
        sigma1 = sigma0;
        gamma0 = zdiv(delta, rho1);
        sigma0 = zdiv(b1, rho1);
        zc ge = zmul(gamma0, eta);
        for (int64_t i = 0; i < n; ++i) {
            zc c = {vc[2 * i], vc[2 * i + 1]}, a = {wp[2 * i], wp[2 * i + 1]};
            zc d = {wc[2 * i], wc[2 * i + 1]};
            zc r = zdiv(zsub(zsub(c, zmul(rho3, a)), zmul(rho2, d)), rho1);
            wp[2 * i] = r.r; wp[2 * i + 1] = r.i;
            zc xx = {x[2 * i], x[2 * i + 1]};
            xx = zadd(xx, zmul(ge, r));
            x[2 * i] = xx.r; x[2 * i + 1] = xx.i;
        }
        res = zscale(res, zabs(sigma0));
        zc ms = {-sigma0.r, -sigma0.i};
        eta = zmul(ms, eta);
        beta0 = beta1;
        double *t = vc; vc = vp; vp = t;
        t = wc; wc = wp; wp = t;
    }
    if (res_out) *res_out = zabs(res);
    free(v); free(w); free(tmp);
    return iter;
}

/* ed_driver.f90:194-248: density matrix <c^+_i c_j> of one eigenvector over a sorted basis
 * of ndim states; out is (nv x nv) column-major like the Fortran array denmat(i, j). */
void orc_denmat(int64_t ndim, const int64_t *fock, int nv, const double *vec, double *out) {
    memset(out, 0, sizeof(double) * 2 * (size_t)nv * (size_t)nv);
    for (int64_t icfg = 1; icfg <= ndim; ++icfg) {
        zc vi = {vec[2 * (icfg - 1)], vec[2 * (icfg - 1) + 1]};
        for (int j = 1; j <= nv; ++j) {
            if (btest(fock[icfg - 1], j - 1)) {
                int64_t o = 2 * ((int64_t)(j - 1) + (int64_t)(j - 1) * nv);
                out[o] += vi.r * vi.r + vi.i * vi.i;
            }
        }
        if (zabs(vi) < 1e-10) continue;
        for (int i = 1; i <= nv - 1; ++i) {
            for (int j = i + 1; j <= nv; ++j) {
                if (!btest(fock[icfg - 1], i - 1)) continue;
                int64_t old = fock[icfg - 1], nw; int sgn, tot = 1;
                orc_make_newfock('-', i, old, &nw, &sgn); tot *= sgn; old = nw;
                if (btest(old, j - 1)) continue;
                orc_make_newfock('+', j, old, &nw, &sgn); tot *= sgn;
                int64_t jcfg = orc_binary_search(ndim, fock, nw);
                if (jcfg == -1) continue;
                zc vj = {vec[2 * (jcfg - 1)], vec[2 * (jcfg - 1) + 1]};
                zc cvi = {vi.r, -vi.i}, cvj = {vj.r, -vj.i};
                zc a = zscale(zmul(cvi, vj), (double)tot);
                zc bb = zscale(zmul(cvj, vi), (double)tot);
                int64_t oij = 2 * ((int64_t)(i - 1) + (int64_t)(j - 1) * nv);
                int64_t oji = 2 * ((int64_t)(j - 1) + (int64_t)(i - 1) * nv);
                out[oij] += a.r; out[oij + 1] += a.i;
                out[oji] += bb.r; out[oji + 1] += bb.i;
            }
        }
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
