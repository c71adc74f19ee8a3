"""Python face of the CPU oracle (test infrastructure only).

``libedx_oracle.so`` (oracle/edx_oracle.c) restates the Fortran build, SpMV, Krylov and
MINRES routines in FP64.  This module binds it with ctypes and adds numpy restatements of
the pieces the reference keeps in Python:

* ``spectra_from_poles``   edrixs/plot_spectrum.py:9-61 (continued fraction)
* ``boltz_dist``           edrixs/utils.py:34-73 (k_B = 8.6173303e-5 eV/K)
* small text readers for the input files, written independently of the product's parser
  (src/io.f90:70-512 formats) so that a parser bug cannot hide on both sides.
* ``ed_eigs``              lowest eigenpairs: dense ``numpy.linalg.eigh`` (ZHEEV, as
  src/full_diag.f90:1-33) or ``scipy.sparse.linalg.eigsh`` (ARPACK, as src/arpack.f90).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libedx_oracle.so")
_lib = None

c_i64p = ctypes.POINTER(ctypes.c_int64)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_dp = ctypes.POINTER(ctypes.c_double)


class _Build(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int),
        ("fock_left", c_i64p), ("ndim_left", ctypes.c_int64),
        ("fock_right", c_i64p), ("ndim_right", ctypes.c_int64),
        ("num_val_orbs", ctypes.c_int), ("num_core_orbs", ctypes.c_int),
        ("nhopp", ctypes.c_int), ("hopp_idx", c_i32p), ("hopp_val", c_dp),
        ("ncoul", ctypes.c_int), ("coul_idx", c_i32p), ("coul_val", c_dp),
        ("ham_sign", ctypes.c_double), ("omega_re", ctypes.c_double),
        ("omega_im", ctypes.c_double),
    ]


def build_oracle_lib():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build_oracle_lib()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_binomial.restype = ctypes.c_int64
        L.orc_binomial.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_fock_full_N.restype = ctypes.c_int64
        L.orc_fock_full_N.argtypes = [ctypes.c_int, ctypes.c_int, c_i64p]
        L.orc_binary_search.restype = ctypes.c_int64
        L.orc_binary_search.argtypes = [ctypes.c_int64, c_i64p, ctypes.c_int64]
        L.orc_build_nrows.restype = ctypes.c_int64
        L.orc_build_nrows.argtypes = [ctypes.POINTER(_Build)]
        L.orc_build_count.restype = ctypes.c_int64
        L.orc_build_count.argtypes = [ctypes.POINTER(_Build), c_i64p]
        L.orc_build_fill.restype = ctypes.c_int
        L.orc_build_fill.argtypes = [ctypes.POINTER(_Build), c_i64p, c_i32p, c_dp]
        L.orc_matvec.restype = None
        L.orc_matvec.argtypes = [ctypes.c_int64, c_i64p, c_i32p, c_dp, c_dp, c_dp]
        L.orc_build_krylov.restype = ctypes.c_int
        L.orc_build_krylov.argtypes = [ctypes.c_int64, c_i64p, c_i32p, c_dp, c_dp, ctypes.c_int,
                                       c_dp, c_dp, c_dp]
        L.orc_minres.restype = ctypes.c_int
        L.orc_minres.argtypes = [ctypes.c_int64, c_i64p, c_i32p, c_dp, c_dp, c_dp,
                                 ctypes.c_double, ctypes.c_int, c_dp]
        L.orc_denmat.restype = None
        L.orc_denmat.argtypes = [ctypes.c_int64, c_i64p, ctypes.c_int, c_dp, c_dp]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def num_threads():
    return lib().orc_num_threads()


# ------------------------------------------------------------------------------------
# Fock basis
# ------------------------------------------------------------------------------------

def fock_full_N(norb, N):
    n = lib().orc_fock_full_N(norb, N, None)
    out = np.empty(n, dtype=np.int64)
    lib().orc_fock_full_N(norb, N, _p(out, c_i64p))
    return out


def binary_search(vec, m):
    vec = np.ascontiguousarray(vec, dtype=np.int64)
    return int(lib().orc_binary_search(len(vec), _p(vec, c_i64p), int(m)))


# ------------------------------------------------------------------------------------
# CSR build
# ------------------------------------------------------------------------------------

class CSR:
    """0-based CSR: row_ptr int64[m+1], col int32[nnz], val complex128[nnz]."""

    def __init__(self, row_ptr, col, val, ncols):
        self.row_ptr, self.col, self.val, self.ncols = row_ptr, col, val, ncols

    @property
    def nrows(self):
        return len(self.row_ptr) - 1

    @property
    def nnz(self):
        return int(self.row_ptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row_ptr), shape=(self.nrows, self.ncols))

    def dense(self):
        return self.to_scipy().toarray()


MODE = {"ham_i": 0, "ham_n": 1, "trans_i": 2, "trans_f": 3}


def build_csr(mode, fock_left, hopping, coulomb=None, fock_right=None, num_val_orbs=0,
              num_core_orbs=0, ham_sign=1.0, omega=0j):
    """hopping = (idx int32[n,2] 1-based, val complex128[n]); coulomb likewise with 4 idx."""
    m = MODE[mode] if isinstance(mode, str) else int(mode)
    fl = np.ascontiguousarray(fock_left, dtype=np.int64)
    fr = np.ascontiguousarray(fock_right if fock_right is not None else fock_left, dtype=np.int64)
    hi = np.ascontiguousarray(hopping[0], dtype=np.int32).reshape(-1, 2)
    hv = np.ascontiguousarray(hopping[1], dtype=np.complex128).view(np.float64)
    if coulomb is None:
        ci = np.zeros((0, 4), dtype=np.int32)
        cv = np.zeros(0, dtype=np.complex128).view(np.float64)
    else:
        ci = np.ascontiguousarray(coulomb[0], dtype=np.int32).reshape(-1, 4)
        cv = np.ascontiguousarray(coulomb[1], dtype=np.complex128).view(np.float64)
    b = _Build(m, _p(fl, c_i64p), len(fl), _p(fr, c_i64p), len(fr), num_val_orbs, num_core_orbs,
               len(hi), _p(hi, c_i32p), _p(hv, c_dp), len(ci), _p(ci, c_i32p), _p(cv, c_dp),
               float(ham_sign), float(np.real(omega)), float(np.imag(omega)))
    L = lib()
    nrows = L.orc_build_nrows(ctypes.byref(b))
    row_nnz = np.zeros(nrows, dtype=np.int64)
    L.orc_build_count(ctypes.byref(b), _p(row_nnz, c_i64p))
    row_ptr = np.zeros(nrows + 1, dtype=np.int64)
    np.cumsum(row_nnz, out=row_ptr[1:])
    nnz = int(row_ptr[-1])
    col = np.zeros(nnz, dtype=np.int32)
    val = np.zeros(nnz, dtype=np.complex128)
    L.orc_build_fill(ctypes.byref(b), _p(row_ptr, c_i64p), _p(col, c_i32p),
                     _p(val.view(np.float64), c_dp))
    if m == 0:
        ncols = len(fl)
    elif m == 1:
        ncols = len(fl) * num_core_orbs
    elif m == 2:
        ncols = len(fr)
    else:
        ncols = len(fr) * num_core_orbs
    return CSR(row_ptr, col, val, ncols)


def matvec(csr, x, y=None):
    """y += A x (spmv.f90:73-103); y defaults to zeros."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    if y is None:
        y = np.zeros(csr.nrows, dtype=np.complex128)
    lib().orc_matvec(csr.nrows, _p(csr.row_ptr, c_i64p), _p(csr.col, c_i32p),
                     _p(csr.val.view(np.float64), c_dp), _p(x.view(np.float64), c_dp),
                     _p(y.view(np.float64), c_dp))
    return y


def build_krylov(csr, phi, maxn):
    """lanczos.f90:210-303 -> (alpha[neff], beta[neff], norm, neff)."""
    phi = np.ascontiguousarray(phi, dtype=np.complex128)
    a = np.zeros(maxn)
    b = np.zeros(maxn)
    norm = ctypes.c_double(0)
    neff = lib().orc_build_krylov(csr.nrows, _p(csr.row_ptr, c_i64p), _p(csr.col, c_i32p),
                                  _p(csr.val.view(np.float64), c_dp),
                                  _p(phi.view(np.float64), c_dp), maxn, _p(a, c_dp), _p(b, c_dp),
                                  ctypes.byref(norm))
    return a[:neff], b[:neff], norm.value, neff


def minres(csr, b, tol, maxit):
    """linsys.f90:3-128 -> (x, iterations, |res| estimate)."""
    b = np.ascontiguousarray(b, dtype=np.complex128)
    x = np.zeros_like(b)
    res = ctypes.c_double(0)
    it = lib().orc_minres(csr.nrows, _p(csr.row_ptr, c_i64p), _p(csr.col, c_i32p),
                          _p(csr.val.view(np.float64), c_dp), _p(b.view(np.float64), c_dp),
                          _p(x.view(np.float64), c_dp), float(tol), int(maxit), ctypes.byref(res))
    return x, it, res.value


def denmat(fock, num_val_orbs, vec):
    """ed_driver.f90:194-248 for one eigenvector -> complex (nv, nv), [i, j] = <c+_i c_j>."""
    fock = np.ascontiguousarray(fock, dtype=np.int64)
    vec = np.ascontiguousarray(vec, dtype=np.complex128)
    out = np.zeros((num_val_orbs, num_val_orbs), dtype=np.complex128, order="F")
    lib().orc_denmat(len(fock), _p(fock, c_i64p), num_val_orbs, _p(vec.view(np.float64), c_dp),
                     out.ctypes.data_as(c_dp))
    return np.array(out)


# ------------------------------------------------------------------------------------
# Spectra (plot_spectrum.py:9-61, utils.py:34-73)
# ------------------------------------------------------------------------------------

KB = 8.6173303e-5


def boltz_dist(gs, T):
    gs = np.array(gs, dtype=np.float64)
    beta = 1.0 / (KB * T)
    w = np.exp(-beta * (gs - gs.min()))
    return w / np.sum(w)


def spectra_from_poles(poles, omega_mesh, gamma_mesh, temperature):
    """poles = dict(npoles, eigval, norm, alpha, beta) as read_poles_from_file builds it."""
    omega_mesh = np.asarray(omega_mesh, dtype=np.float64)
    gamma_mesh = np.broadcast_to(np.asarray(gamma_mesh, dtype=np.float64), omega_mesh.shape)
    spec = np.zeros(len(omega_mesh))
    w = boltz_dist(poles["eigval"], temperature)
    for i in range(len(poles["eigval"])):
        neff = poles["npoles"][i]
        a, b = poles["alpha"][i], poles["beta"][i]
        e0, nrm = poles["eigval"][i], poles["norm"][i]
        t = np.zeros(len(omega_mesh), dtype=complex)
        for j in range(neff - 1, 0, -1):
            t = b[j - 1] ** 2 / (omega_mesh + 1j * gamma_mesh + e0 - a[j] - t)
        t = 1.0 / (omega_mesh + 1j * gamma_mesh + e0 - a[0] - t)
        spec += -1.0 / np.pi * np.imag(t) * nrm * w[i]
    return spec


# ------------------------------------------------------------------------------------
# Independent text readers (src/io.f90 formats)
# ------------------------------------------------------------------------------------

def read_terms(path, nidx):
    with open(path) as f:
        n = int(f.readline().split()[0])
        rows = [f.readline().split() for _ in range(n)]
    idx = np.array([[int(r[k]) for k in range(nidx)] for r in rows], dtype=np.int32).reshape(-1, nidx)
    val = np.array([float(r[nidx]) + 1j * float(r[nidx + 1]) for r in rows], dtype=np.complex128)
    return idx, val


def read_fock(path):
    with open(path) as f:
        n = int(f.readline().split()[0])
        data = np.array([int(f.readline()) for _ in range(n)], dtype=np.int64)
    return data


# ------------------------------------------------------------------------------------
# Eigen-solvers used as the ED oracle
# ------------------------------------------------------------------------------------

def ed_eigs(csr, nev, dense_below=3000, tol=1e-13):
    """Lowest nev eigenpairs (ascending).  Dense ZHEEV-equivalent below `dense_below`."""
    n = csr.nrows
    if n <= dense_below:
        h = csr.dense()
        e, v = np.linalg.eigh(h)
        return e[:nev], v[:, :nev]
    import scipy.sparse.linalg as sla
    e, v = sla.eigsh(csr.to_scipy(), k=nev, which="SA", tol=tol, ncv=max(2 * nev + 20, 40))
    order = np.argsort(e)
    return e[order], v[:, order]


def _tridiag_eigs(alpha, beta):
    """krylov_eigs (src/lanczos.f90:169-206): dsteqr('I') on the i x i tridiagonal matrix.
    LAPACK's dstev with vectors runs the same implicit QL/QR (dsteqr)."""
    from scipy.linalg import lapack
    d, z, info = lapack.dstev(np.asarray(alpha, dtype=np.float64), np.asarray(beta, dtype=np.float64),
                              compute_v=1)
    if info != 0:
        raise RuntimeError(f"dstev info {info}")
    return d, z


def lanczos_eigs(csr, nev, max_niter, eval_tol, nvec=1, seed=0):
    """diag_ham_lanczos (src/lanczos.f90:6-167), the ed_solver = 1 path of ed_driver.f90:154-158.

    Plain Lanczos without reorthogonalisation, step for step:
    * start vector: uniform reals in [-0.5, 0.5), zero imaginary part, normalised
      (:60-70). The reference calls random_seed() without arguments, so its start vector is
      processor-dependent; here it is numpy's default generator with `seed`.
    * step i: w = H v_i - beta_{i-1} v_{i-1}; alpha_i = Re<v_i, w> (:76-88).
    * every 10th step and at max_niter: eigenvalues of T_i (dsteqr); once i >= nev, stop when
      |lambda_nev(T_i) - lambda_nev(previous check)| < eval_tol (:89-110). The previous check
      starts at 0.
    * w -= alpha_i v_i; beta_i = |w|; stop when beta_i < 1e-10 (:111-131).
    * eigenvectors: the recurrence is run again from the stored start vector and
      sum_i z_ij v_i accumulated over the nkrylov steps (:133-157). When max_niter passes
      without convergence nkrylov stays 0 and the eigenvectors are zero, as in the reference.
    Where T_i is smaller than nev, the missing eigenvalues read the zeroed work array and are 0.
    Returns (eval[nev], evec[n, nvec], nkrylov).
    """
    n = csr.nrows
    rng = np.random.default_rng(seed)
    v1 = (rng.random(n) - 0.5).astype(np.complex128)
    v1 /= np.sqrt(np.vdot(v1, v1).real)
    alpha = np.zeros(max_niter)
    beta = np.zeros(max_niter + 1)                     # beta[0] is beta(0) = 0
    evals = np.zeros(nev)
    kvec = None
    nkrylov = 0
    curr, prev = v1.copy(), np.zeros(n, dtype=np.complex128)
    for i in range(1, max_niter + 1):
        prev = -beta[i - 1] * prev
        prev = matvec(csr, curr, prev)
        alpha[i - 1] = np.vdot(curr, prev).real
        if i % 10 == 0 or i == max_niter:
            ke, kv = _tridiag_eigs(alpha[:i], beta[1:i])
            ke = np.concatenate([ke, np.zeros(max(0, nev - i))])
            if i >= nev:
                if abs(ke[nev - 1] - evals[nev - 1]) < eval_tol:
                    evals = ke[:nev].copy()
                    nkrylov, kvec = i, kv
                    break
            evals = ke[:nev].copy()
        prev = prev - alpha[i - 1] * curr
        beta[i] = np.sqrt(np.vdot(prev, prev).real)
        if abs(beta[i]) < 1e-10:
            if i >= 2:
                ke, kvec = _tridiag_eigs(alpha[:i], beta[1:i])
                ke = np.concatenate([ke, np.zeros(max(0, nev - i))])
                evals = ke[:nev].copy()
            else:
                evals[0] = alpha[0]
                kvec = np.ones((1, 1))
            nkrylov = i
            break
        prev = prev / beta[i]
        curr, prev = prev, curr
    evec = np.zeros((n, nvec), dtype=np.complex128)
    curr, prev = v1.copy(), np.zeros(n, dtype=np.complex128)
    for i in range(1, nkrylov + 1):
        m = min(nvec, kvec.shape[1])
        evec[:, :m] += np.outer(curr, kvec[i - 1, :m])
        if i < nkrylov:
            prev = -alpha[i - 1] * curr - beta[i - 1] * prev
            prev = matvec(csr, curr, prev)
            prev = prev / beta[i]
            curr, prev = prev, curr
    return evals, evec, nkrylov
