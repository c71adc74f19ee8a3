"""Oracle ED / XAS / RIXS drivers (test infrastructure only).

They restate src/ed_driver.f90, src/xas_driver.f90 and src/rixs_driver.f90 on top of the C
oracle (build, SpMV, Krylov, MINRES) and read the same input files, so that the drop-in
solvers of edrixs_b200.fedrixs and the batched RIXS path can be checked against them.
Eigenpairs come from dense ZHEEV-equivalent numpy (small) or scipy ARPACK (larger), which
is what the reference's ed_solver = 0 / 2 paths compute.
"""
import os

import numpy as np

from . import pyoracle as orc


def _cfg(path):
    import re
    txt = open(path).read()
    body = re.search(r"&control(.*?)&end", txt, flags=re.S | re.I).group(1)
    cfg = {"ed_solver": 1, "num_val_orbs": 2, "num_core_orbs": 2, "neval": 1, "nvector": 1, "idump": False,
           "num_gs": 1, "maxiter": 500, "linsys_max": 500, "min_ndim": 1000, "eigval_tol": 1e-8,
           "linsys_tol": 1e-8, "nkryl": 500, "omega_in": 0.0, "gamma_in": 0.1}
    for k, v in re.findall(r"(\w+)\s*=\s*([^,\n]+)", body):
        k = k.lower()
        v = v.strip()
        if k == "idump":
            cfg[k] = v.lower().strip(".").startswith("t")
        elif k in ("eigval_tol", "linsys_tol", "omega_in", "gamma_in"):
            cfg[k] = float(v.lower().replace("d", "e"))
        else:
            cfg[k] = int(float(v))
    return cfg


def ed(directory, follow_ed_solver=False):
    """-> eigvals (neval), eigvecs (n, nvector), H csr, fock, cfg.  By default the eigenpairs
    are those of ed_solver 0 / 2 (dense or ARPACK).  With follow_ed_solver, ed_solver = 1 at
    or above min_ndim runs the step-for-step plain Lanczos of lanczos.f90:6-167 instead, as
    ed_driver.f90:154-158 does (seeded; lowest distinct levels on degenerate spectra)."""
    p = lambda f: os.path.join(directory, f)  # noqa: E731
    cfg = _cfg(p("config.in"))
    fock = orc.read_fock(p("fock_i.in"))
    H = orc.build_csr("ham_i", fock, orc.read_terms(p("hopping_i.in"), 2), orc.read_terms(p("coulomb_i.in"), 4),
                      num_val_orbs=cfg["num_val_orbs"])
    neval = min(cfg["neval"], len(fock))
    nvec = min(cfg["nvector"], len(fock))
    if follow_ed_solver and cfg["ed_solver"] == 1 and len(fock) >= cfg["min_ndim"]:
        e, v, _ = orc.lanczos_eigs(H, neval, cfg["maxiter"], cfg["eigval_tol"], nvec=nvec)
        return e, v, H, fock, cfg
    e, v = orc.ed_eigs(H, max(neval, nvec))
    return e[:neval], v[:, :nvec], H, fock, cfg


def denmat(fock, nv, vecs):
    return np.stack([orc.denmat(fock, nv, vecs[:, k]) for k in range(vecs.shape[1])])


def read_eigvec(path):
    import struct
    raw = open(path, "rb").read()
    (n1,) = struct.unpack_from("<i", raw, 0)
    e = struct.unpack_from("<d", raw, 4)[0]
    off = 4 + n1 + 4
    (n2,) = struct.unpack_from("<i", raw, off)
    v = np.frombuffer(raw[off + 4: off + 4 + n2], dtype=np.complex128).copy()
    return e, v


def xas(directory):
    """-> list of (alpha, beta, norm, neff, e_gs) per ground state (xas_driver.f90:65-155)."""
    p = lambda f: os.path.join(directory, f)  # noqa: E731
    cfg = _cfg(p("config.in"))
    nv, nc = cfg["num_val_orbs"], cfg["num_core_orbs"]
    fi, fn = orc.read_fock(p("fock_i.in")), orc.read_fock(p("fock_n.in"))
    D = orc.build_csr("trans_i", fn, orc.read_terms(p("transop_xas.in"), 2), fock_right=fi, num_val_orbs=nv,
                      num_core_orbs=nc)
    Hn = orc.build_csr("ham_n", fn, orc.read_terms(p("hopping_n.in"), 2), orc.read_terms(p("coulomb_n.in"), 4),
                       num_val_orbs=nv, num_core_orbs=nc)
    out = []
    for igs in range(1, cfg["num_gs"] + 1):
        e, g = read_eigvec(p(f"eigvec.{igs}"))
        phi = orc.matvec(D, g)
        a, b, nrm, neff = orc.build_krylov(Hn, phi, cfg["nkryl"])
        out.append((a, b, nrm, neff, e))
    return out


def rixs(directory):
    """-> list of (alpha, beta, norm, neff, e_gs, minres_iters) per ground state
    (rixs_driver.f90:73-231, A built explicitly with ham_sign = -1 and omega)."""
    p = lambda f: os.path.join(directory, f)  # noqa: E731
    cfg = _cfg(p("config.in"))
    nv, nc = cfg["num_val_orbs"], cfg["num_core_orbs"]
    fi, fn, ff = orc.read_fock(p("fock_i.in")), orc.read_fock(p("fock_n.in")), orc.read_fock(p("fock_f.in"))
    Din = orc.build_csr("trans_i", fn, orc.read_terms(p("transop_rixs_i.in"), 2), fock_right=fi, num_val_orbs=nv,
                        num_core_orbs=nc)
    Dout = orc.build_csr("trans_f", ff, orc.read_terms(p("transop_rixs_f.in"), 2), fock_right=fn, num_val_orbs=nv,
                         num_core_orbs=nc)
    hop_n, coul_n = orc.read_terms(p("hopping_n.in"), 2), orc.read_terms(p("coulomb_n.in"), 4)
    Hf = orc.build_csr("ham_i", ff, orc.read_terms(p("hopping_i.in"), 2), orc.read_terms(p("coulomb_i.in"), 4),
                       num_val_orbs=nv)
    out = []
    for igs in range(1, cfg["num_gs"] + 1):
        e, g = read_eigvec(p(f"eigvec.{igs}"))
        phi = orc.matvec(Din, g)
        A = orc.build_csr("ham_n", fn, hop_n, coul_n, num_val_orbs=nv, num_core_orbs=nc, ham_sign=-1.0,
                          omega=complex(cfg["omega_in"] + e, cfg["gamma_in"]))
        x, it, res = orc.minres(A, phi, cfg["linsys_tol"], cfg["linsys_max"])
        phi_f = orc.matvec(Dout, x)
        a, b, nrm, neff = orc.build_krylov(Hf, phi_f, cfg["nkryl"])
        out.append((a, b, nrm, neff, e, it))
    return out


def opavg(directory):
    """-> (eigvals, <v|O|v>) per eigvec.N, N = 1..num_gs (src/opavg_driver.f90:62-112): O is
    built from hopping_i.in / coulomb_i.in on fock_i.in as build_ham_i builds a Hamiltonian,
    then dot_product(v, O v) (:103-106)."""
    p = lambda f: os.path.join(directory, f)  # noqa: E731
    cfg = _cfg(p("config.in"))
    fock = orc.read_fock(p("fock_i.in"))
    O = orc.build_csr("ham_i", fock, orc.read_terms(p("hopping_i.in"), 2), orc.read_terms(p("coulomb_i.in"), 4),
                      num_val_orbs=cfg["num_val_orbs"])
    ev, avg = [], []
    for igs in range(1, cfg["num_gs"] + 1):
        e, v = read_eigvec(p(f"eigvec.{igs}"))
        ev.append(e)
        avg.append(np.vdot(v, orc.matvec(O, v)))
    return np.array(ev), np.array(avg)


def rixs_in_memory(terms, nv, nelec, gs_e, gs_v, din_terms, dout_terms, omegas, gamma_c, eloss, gamma_f, nkryl,
                   tol, maxit, temperature):
    """The reference's loop (solvers.py:2651-2702) for every omega x pol pair x ground state;
    -> spectra (n_omega, n_eloss, n_pin * n_pout) ordered (pol_in, pol_out)."""
    fi = orc.fock_full_N(nv, nelec)
    fn = orc.fock_full_N(nv, nelec + 1)
    Hn = orc.build_csr("ham_n", fn, terms["hop_n"], terms["coul_n"], num_val_orbs=nv, num_core_orbs=6)
    Hf = orc.build_csr("ham_i", fi, terms["hop_i"], terms["coul_i"], num_val_orbs=nv)
    Din = [orc.build_csr("trans_i", fn, t, fock_right=fi, num_val_orbs=nv, num_core_orbs=6) for t in din_terms]
    Dout = [orc.build_csr("trans_f", fi, t, fock_right=fn, num_val_orbs=nv, num_core_orbs=6) for t in dout_terms]
    import scipy.sparse as sp
    Hs = Hn.to_scipy()
    I = sp.identity(Hn.nrows, format="csr", dtype=np.complex128)
    out = np.zeros((len(omegas), len(eloss), len(Din) * len(Dout)))
    for w, om in enumerate(omegas):
        for pi, D in enumerate(Din):
            xs = []
            for g in range(len(gs_e)):
                phi = orc.matvec(D, gs_v[:, g])
                M = (complex(om + gs_e[g], gamma_c) * I - Hs).tocsr()
                M.sort_indices()
                A = orc.CSR(M.indptr.astype(np.int64), M.indices.astype(np.int32), M.data.astype(np.complex128),
                            M.shape[1])
                x, it, res = orc.minres(A, phi, tol, maxit)
                xs.append(x)
            for po, Do in enumerate(Dout):
                poles = {"npoles": [], "eigval": [], "norm": [], "alpha": [], "beta": []}
                for g in range(len(gs_e)):
                    a, b, nrm, neff = orc.build_krylov(Hf, orc.matvec(Do, xs[g]), nkryl)
                    poles["npoles"].append(neff)
                    poles["eigval"].append(gs_e[g])
                    poles["norm"].append(nrm)
                    poles["alpha"].append(list(a))
                    poles["beta"].append(list(b))
                out[w, :, pi * len(Dout) + po] = orc.spectra_from_poles(poles, eloss, gamma_f, temperature)
    return out
