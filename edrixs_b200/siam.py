"""Seeded single-impurity Anderson model (SIAM) inputs for the ED/XAS/RIXS workloads.

Restates the emat/umat assembly of ``ed_siam_fort`` (edrixs/solvers.py:2012-2135, general
hopping form ``siam_type=1`` at :2032-2038) for a 3d impurity (10 spin-orbitals, orbitals
1-10), ``nbath`` bath spin-orbitals (11..10+nbath) and a 2p core shell (6 spin-orbitals,
placed after the valence orbitals, as docs/user_guide.lyx:1903-1948 requires).  The atomic
tensors (Slater unit tensors, spin-orbit matrices, dipole operators, polarisation vectors)
are the reference's own outputs, captured once in ``data/atomic_dp.npz``.

Draw order of ``numpy.random.default_rng(seed)`` (fixed, so every size is reproducible):
  1. crystal field: 10 values U(-0.5, 0.5) eV on the impurity diagonal;
  2. bath levels: nbath values U(-3, 3) eV;
  3. hybridisation V (10 x nbath): Re ~ N(0, sigma=0.5), then Im ~ N(0, sigma=0.5),
     placed Hermitian (V in the impurity-bath block, V^H in the bath-impurity block).
"""
import os
from dataclasses import dataclass, field

import numpy as np

from . import io as edxio

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "atomic_dp.npz")
_atomic = None

# core-valence Slater integrals of the intermediate (core-hole) Hamiltonian.  The workloads
# fix F0/F2/F4 of the d shell and the core spin-orbit coupling; these are chosen here.
DEFAULT_SLATER_VC = (7.5, 6.0, 4.5, 2.6)  # F0_dp, F2_dp, G1_dp, G3_dp (eV)
KB = 8.6173303e-5


def atomic():
    global _atomic
    if _atomic is None:
        with np.load(_DATA) as z:
            _atomic = {k: z[k] for k in z.files}
    return _atomic


def _umat_from_units(prefix, coeffs, norb):
    a = atomic()
    u = np.zeros((norb,) * 4, dtype=np.complex128)
    for k, c in enumerate(coeffs):
        if c == 0.0:
            continue
        idx = a[f"{prefix}_unit{k}_idx"].astype(np.int64)
        u[tuple(idx.T)] += c * a[f"{prefix}_unit{k}_val"]
    return u


def umat_slater_dp(slater):
    """get_umat_slater('dp', F0_dd, F2_dd, F4_dd, F0_dp, F2_dp, G1_dp, G3_dp, F0_pp, F2_pp)."""
    coeffs = list(slater) + [0.0] * (9 - len(slater))
    return _umat_from_units("umat_dp", coeffs, 16)


def umat_slater_d(F0, F2, F4):
    return _umat_from_units("umat_d", (F0, F2, F4), 10)


@dataclass
class SiamModel:
    nbath: int
    nelec: int
    seed: int
    emat_i: np.ndarray
    emat_n: np.ndarray
    umat_i: np.ndarray
    umat_n: np.ndarray
    trans_op: np.ndarray            # (3, ntot, ntot) dipole operators, valence x core block
    meta: dict = field(default_factory=dict)

    @property
    def nv(self):
        return 10 + self.nbath

    @property
    def ntot(self):
        return self.nv + 6


def make_siam(nbath, nelec, seed, slater_i=(8.0, 10.0, 6.2), slater_vc=DEFAULT_SLATER_VC, zeta_v=0.08,
              zeta_c=11.0, c_level=0.0):
    """Build the SIAM tensors for 10 impurity + nbath bath valence orbitals and a 2p core."""
    a = atomic()
    rng = np.random.default_rng(seed)
    cf = rng.uniform(-0.5, 0.5, 10)
    bath = rng.uniform(-3.0, 3.0, nbath)
    V = rng.normal(0.0, 0.5, (10, nbath)) + 1j * rng.normal(0.0, 0.5, (10, nbath))
    nv = 10 + nbath
    ntot = nv + 6
    hop = np.zeros((nv, nv), dtype=np.complex128)
    hop[:10, :10] = zeta_v * a["hsoc_d_unit"] + np.diag(cf)
    hop[10:, 10:] = np.diag(bath)
    hop[:10, 10:] = V
    hop[10:, :10] = V.conj().T
    emat_i = np.zeros((ntot, ntot), dtype=np.complex128)
    emat_n = np.zeros((ntot, ntot), dtype=np.complex128)
    emat_i[:nv, :nv] = hop
    emat_n[:nv, :nv] = hop
    emat_n[nv:, nv:] = zeta_c * a["hsoc_p_unit"] + c_level * np.eye(6)
    # place the (10 d + 6 p) Slater tensor on orbitals [0..9] + [nv..nv+5] (solvers.py:2017-2025)
    idx = np.array(list(range(10)) + [nv + i for i in range(6)])
    u_i = umat_slater_dp(tuple(slater_i))
    u_n = umat_slater_dp(tuple(slater_i) + tuple(slater_vc))
    umat_i = np.zeros((ntot,) * 4, dtype=np.complex128)
    umat_n = np.zeros((ntot,) * 4, dtype=np.complex128)
    ix = np.ix_(idx, idx, idx, idx)
    umat_i[ix] = u_i
    umat_n[ix] = u_n
    trans = np.zeros((3, ntot, ntot), dtype=np.complex128)
    trans[:, :10, nv:] = a["trans_oper_dp"]
    return SiamModel(nbath, nelec, seed, emat_i, emat_n, umat_i, umat_n, trans,
                     meta=dict(slater_i=tuple(slater_i), slater_vc=tuple(slater_vc), zeta_v=zeta_v,
                               zeta_c=zeta_c, c_level=c_level))


def polarised_operator(model, polvec):
    """sum_i polvec_i T_i (solvers.py:2441-2443 / :2678-2685)."""
    return np.tensordot(np.asarray(polvec, dtype=np.complex128), model.trans_op, axes=(0, 0))


def rixs_polarisations():
    """(pol_in, pol_out) vectors for linear pi/sigma in and out (thin=15, thout=75 deg)."""
    a = atomic()
    return [(a["rixs_polvec_in"][p], a["rixs_polvec_out"][p]) for p in range(4)]


def nonzero_terms(t, tol=1e-12):
    """(1-based idx, value) of |t| > tol in row-major order, as write_emat/write_umat emit them."""
    nz = np.nonzero(np.abs(t) > tol)
    idx = np.stack(nz, axis=-1).astype(np.int32) + 1
    val = t[nz].astype(np.complex128)
    if len(val) == 0:  # the reference writes a single zero term "1 1 0 0"
        idx = np.ones((1, t.ndim), dtype=np.int32)
        val = np.zeros(1, dtype=np.complex128)
    return idx, val


def text_roundtrip(terms, nidx):
    """Values exactly as they come back from the '{:.15f}' text of write_emat/write_umat."""
    idx, val = terms
    re = np.array([float("{:.15f}".format(v)) for v in val.real])
    im = np.array([float("{:.15f}".format(v)) for v in val.imag])
    return idx, re + 1j * im


def write_ed_inputs(model, directory, *, neval=1, nvector=1, ed_solver=2, ncv=None, idump=True, maxiter=1000,
                    eigval_tol=1e-10, min_ndim=1000, write_fock=True):
    """Files ed_siam_fort writes before ed_fsolver (solvers.py:2126-2136)."""
    os.makedirs(directory, exist_ok=True)
    edxio.write_umat(model.umat_i, os.path.join(directory, "coulomb_i.in"))
    edxio.write_umat(model.umat_n, os.path.join(directory, "coulomb_n.in"))
    edxio.write_emat(model.emat_i, os.path.join(directory, "hopping_i.in"))
    edxio.write_emat(model.emat_n, os.path.join(directory, "hopping_n.in"))
    edxio.write_config(directory, ed_solver=ed_solver, num_val_orbs=model.nv, neval=neval, nvector=nvector,
                       ncv=ncv if ncv is not None else neval + 2, idump=idump, maxiter=maxiter,
                       min_ndim=min_ndim, eigval_tol=eigval_tol)
    if write_fock:
        edxio.write_fock(os.path.join(directory, "fock_i.in"), fock_states(model.nv, model.nelec))


def fock_states(norb, nelec):
    """Ascending norb-bit states with nelec bits (host-side, for writing fock_*.in)."""
    from itertools import combinations
    out = np.fromiter((sum(1 << b for b in c) for c in combinations(range(norb), nelec)), dtype=np.uint64)
    out.sort()
    return out


def write_xas_inputs(model, directory, polvec, num_gs=1, nkryl=200):
    os.makedirs(directory, exist_ok=True)
    edxio.write_config(directory, num_val_orbs=model.nv, num_core_orbs=6, num_gs=num_gs, nkryl=nkryl)
    edxio.write_fock(os.path.join(directory, "fock_i.in"), fock_states(model.nv, model.nelec))
    edxio.write_fock(os.path.join(directory, "fock_n.in"), fock_states(model.nv, model.nelec + 1))
    edxio.write_emat(polarised_operator(model, polvec), os.path.join(directory, "transop_xas.in"))


def write_rixs_inputs(model, directory, pol_in, pol_out, omega_in, gamma_in, num_gs=1, nkryl=150,
                      linsys_max=1000, linsys_tol=1e-10):
    os.makedirs(directory, exist_ok=True)
    edxio.write_config(directory, num_val_orbs=model.nv, num_core_orbs=6, omega_in=omega_in, gamma_in=gamma_in,
                       num_gs=num_gs, nkryl=nkryl, linsys_max=linsys_max, linsys_tol=linsys_tol)
    edxio.write_fock(os.path.join(directory, "fock_i.in"), fock_states(model.nv, model.nelec))
    edxio.write_fock(os.path.join(directory, "fock_n.in"), fock_states(model.nv, model.nelec + 1))
    edxio.write_fock(os.path.join(directory, "fock_f.in"), fock_states(model.nv, model.nelec))
    edxio.write_emat(polarised_operator(model, pol_in), os.path.join(directory, "transop_rixs_i.in"))
    edxio.write_emat(np.conj(polarised_operator(model, pol_out)).T, os.path.join(directory, "transop_rixs_f.in"))
