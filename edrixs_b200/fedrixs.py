"""Drop-in replacement of the reference's f2py module ``edrixs.fedrixs``.

``ed_fsolver``, ``xas_fsolver``, ``rixs_fsolver`` and ``opavg_fsolver`` keep the signature
``(comm, my_id, num_procs)`` of src/pyapi.f90:1,58,120,184 and the file contract of the
Fortran drivers: inputs from the working directory (config.in, hopping_*.in,
coulomb_*.in, fock_*.in, transop_*.in, eigvec.N), outputs eigvals.dat, denmat.dat,
eigvec.N, xas_poles.N, rixs_poles.N, opavg.dat.  All numerical work runs on the current
CUDA device through libedx; rank 0 does it alone (the Hilbert space is not split across
processes), the other ranks return immediately -- the reference's communicator split of
pyapi.f90:28-48 generalised to "only rank 0 has work".

To use it under the reference's Python layer, make ``edrixs.fedrixs`` resolve to this
module (``sys.modules['edrixs.fedrixs'] = edrixs_b200.fedrixs``, or an ``edrixs/fedrixs.py``
shim that re-exports these four names).  A fake single-rank communicator such as
``FakeComm`` below lets solvers.py run without mpi4py.
"""
import os

import numpy as np
import torch

from . import device
from . import io as edxio
from . import solvers, trace


class FakeComm:
    """The calls edrixs/solvers.py makes on an mpi4py communicator, for one process."""

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def py2f(self):
        return 0

    def Barrier(self):
        pass


def _path(name):
    return os.path.join(os.getcwd(), name)


def ed_core(cfg, H):
    """Lowest eigenpairs of H as src/ed_driver.f90:65-181 chooses them from config.in's
    ed_solver / min_ndim / neval / nvector / eigval_tol: (eigvals, eigvecs (n, nvector))."""
    ndim = H.nrows
    ed_solver = cfg["ed_solver"]
    if ndim < cfg["min_ndim"]:
        ed_solver = 0
    elif ed_solver not in (1, 2):
        # the reference has no branch for other values and writes unset eigenvalues
        # (src/ed_driver.f90:127-171)
        raise edxio.EdxInputError(f"config.in: ed_solver must be 0, 1 or 2 (got {ed_solver})")
    neval = min(cfg["neval"], ndim)
    nvector = min(cfg["nvector"], ndim)
    if ed_solver == 0:
        e, v = solvers.dense_eigs(H, max(neval, nvector))
        return e[:neval], v[:, :nvector]
    if ed_solver == 1:
        # the reference's plain Lanczos (src/lanczos.f90:6-167): its stopping rule, and on a
        # degenerate spectrum its lowest distinct levels
        return solvers.plain_lanczos_eigs(H, neval, nvector, cfg["maxiter"], float(cfg["eigval_tol"]),
                                          packed=device.pack(H))
    tol = min(float(cfg["eigval_tol"]), 1e-9)
    # ARPACK's place (src/arpack.f90:2-112): block thick-restart Lanczos; products on the
    # packed form when H has few enough distinct values (lossless)
    e, v = solvers.lowest_eigs(H, neval, nvector, tol=tol, packed=device.pack(H))
    return e, v


def ed_fsolver(comm=0, my_id=0, num_procs=1):
    """src/ed_driver.f90: build H_i, lowest eigenpairs, eigvals.dat, denmat.dat, eigvec.N."""
    if my_id != 0:
        return
    device.require_cuda()
    cfg = edxio.read_config(_path("config.in"))
    hop = edxio.read_hopping(_path("hopping_i.in"))
    coul = edxio.read_coulomb(_path("coulomb_i.in"))
    fock = edxio.read_fock(_path("fock_i.in"))
    basis = device.basis_from_states(fock)
    with trace.phase("ed: build H_i"):
        H = device.build_csr(device.HAM_I, basis, hop, coul, num_val_orbs=cfg["num_val_orbs"])
    with trace.phase("ed: eigenpairs"):
        e, v = ed_core(cfg, H)
    edxio.write_eigvals(_path("eigvals.dat"), e)
    nv = cfg["num_val_orbs"]
    with trace.phase("ed: density matrix"):
        dm = device.denmat(basis, nv, v).cpu().numpy()
    edxio.write_denmat(_path("denmat.dat"), dm)
    if cfg["idump"]:
        vh = v.cpu().numpy()
        for k in range(vh.shape[1]):
            edxio.write_eigvec(_path(f"eigvec.{k + 1}"), e[k] if k < len(e) else 0.0, vh[:, k])
    torch.cuda.synchronize()


def _read_gs(num_gs, ndim):
    evals, vecs = [], []
    for igs in range(1, num_gs + 1):
        e, v = edxio.read_eigvec(_path(f"eigvec.{igs}"), ndim)
        evals.append(e)
        vecs.append(v)
    return np.array(evals), np.stack(vecs, axis=1)


def xas_fsolver(comm=0, my_id=0, num_procs=1):
    """src/xas_driver.f90: per ground state, D|g>, Krylov of H_n, xas_poles.N.  All ground
    states run as columns of one Krylov block (one SpMM per iteration)."""
    if my_id != 0:
        return
    device.require_cuda()
    cfg = edxio.read_config(_path("config.in"))
    hop_n = edxio.read_hopping(_path("hopping_n.in"))
    coul_n = edxio.read_coulomb(_path("coulomb_n.in"))
    trans = edxio.read_hopping(_path("transop_xas.in"))
    fi = device.basis_from_states(edxio.read_fock(_path("fock_i.in")))
    fn = device.basis_from_states(edxio.read_fock(_path("fock_n.in")))
    nv, nc = cfg["num_val_orbs"], cfg["num_core_orbs"]
    num_gs = cfg["num_gs"]
    evals, g = _read_gs(num_gs, fi.ndim)
    with trace.phase("xas: D|g>"):
        D = device.build_csr(device.TRANS_I, fn, trans, right=fi, num_val_orbs=nv, num_core_orbs=nc)
        phi = device.spmm(D, torch.from_numpy(g).cuda())
    with trace.phase("xas: build H_n"):
        Hn = device.build_csr(device.HAM_N, fn, hop_n, coul_n, num_val_orbs=nv, num_core_orbs=nc)
    with trace.phase("xas: Krylov"):
        r = device.krylov(Hn, phi, cfg["nkryl"])
    _write_poles("xas_poles", r, evals)


def _write_poles(prefix, r, evals):
    a, b = r.alpha.cpu().numpy(), r.beta.cpu().numpy()
    nrm, neff = r.norm.cpu().numpy(), r.neff.cpu().numpy()
    for igs in range(len(evals)):
        ne = int(neff[igs])
        edxio.write_poles(_path(f"{prefix}.{igs + 1}"), ne, a[igs, :ne], b[igs, :ne], float(nrm[igs]),
                          float(evals[igs]))


def rixs_fsolver(comm=0, my_id=0, num_procs=1):
    """src/rixs_driver.f90 for one (omega_in, polarisation pair): per ground state, D_in|g>,
    MINRES on (omega_in + E_g + i*gamma_in - H_n), D_out^+ x, Krylov of H_f, rixs_poles.N.
    The operator omega + E_g + i*gamma - H_n is applied to one resident H_n (alpha = -1,
    sigma = z) instead of rebuilding it per ground state; the final-state Krylov runs all
    ground states as one block."""
    if my_id != 0:
        return
    device.require_cuda()
    cfg = edxio.read_config(_path("config.in"))
    hop_i = edxio.read_hopping(_path("hopping_i.in"))
    coul_i = edxio.read_coulomb(_path("coulomb_i.in"))
    hop_n = edxio.read_hopping(_path("hopping_n.in"))
    coul_n = edxio.read_coulomb(_path("coulomb_n.in"))
    tr_i = edxio.read_hopping(_path("transop_rixs_i.in"))
    tr_f = edxio.read_hopping(_path("transop_rixs_f.in"))
    fi = device.basis_from_states(edxio.read_fock(_path("fock_i.in")))
    fn = device.basis_from_states(edxio.read_fock(_path("fock_n.in")))
    ff = device.basis_from_states(edxio.read_fock(_path("fock_f.in")))
    nv, nc = cfg["num_val_orbs"], cfg["num_core_orbs"]
    num_gs = cfg["num_gs"]
    evals, g = _read_gs(num_gs, fi.ndim)
    with trace.phase("rixs: D_in|g>"):
        Din = device.build_csr(device.TRANS_I, fn, tr_i, right=fi, num_val_orbs=nv, num_core_orbs=nc)
        phi = device.spmm(Din, torch.from_numpy(g).cuda())
    with trace.phase("rixs: build H_n"):
        Hn = device.build_csr(device.HAM_N, fn, hop_n, coul_n, num_val_orbs=nv, num_core_orbs=nc)
    xs = []
    with trace.phase("rixs: MINRES"):
        for igs in range(num_gs):
            z = complex(cfg["omega_in"] + evals[igs], cfg["gamma_in"])
            x, it, res = device.minres(Hn, phi[:, igs].contiguous(), cfg["linsys_tol"], cfg["linsys_max"],
                                       alpha=-1.0, sigma=z)
            xs.append(x)
    X = torch.stack(xs, dim=1)
    with trace.phase("rixs: D_out^+ x"):
        Dout = device.build_csr(device.TRANS_F, ff, tr_f, right=fn, num_val_orbs=nv, num_core_orbs=nc)
        phi_f = device.spmm(Dout, X)
    with trace.phase("rixs: build H_f"):
        Hf = device.build_csr(device.HAM_I, ff, hop_i, coul_i, num_val_orbs=nv)
    with trace.phase("rixs: Krylov"):
        r = device.krylov(Hf, phi_f, cfg["nkryl"])
    _write_poles("rixs_poles", r, evals)


def opavg_fsolver(comm=0, my_id=0, num_procs=1):
    """src/opavg_driver.f90: <v|O|v> of the eigenvectors eigvec.N for the operator given by
    hopping_i.in / coulomb_i.in, written to opavg.dat."""
    if my_id != 0:
        return
    device.require_cuda()
    cfg = edxio.read_config(_path("config.in"))
    hop = edxio.read_hopping(_path("hopping_i.in"))
    coul = edxio.read_coulomb(_path("coulomb_i.in"))
    fi = device.basis_from_states(edxio.read_fock(_path("fock_i.in")))
    evals, g = _read_gs(cfg["num_gs"], fi.ndim)
    with trace.phase("opavg: build O, <v|O|v>"):
        O = device.build_csr(device.HAM_I, fi, hop, coul, num_val_orbs=cfg["num_val_orbs"])
        G = torch.from_numpy(g).cuda()
        OG = device.spmm(O, G)
        avg = (G.conj() * OG).sum(dim=0).cpu().numpy()
    edxio.write_opavg(_path("opavg.dat"), evals, avg)
