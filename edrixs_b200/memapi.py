"""In-memory forms of the reference's single-impurity callers: the same tensors in, the same
results out, no text files.

The reference's ed_siam_fort, xas_siam_fort and rixs_siam_fort (edrixs/solvers.py:1819,
:2268, :2478) turn their physical parameters into a one-body matrix emat, a Coulomb tensor
umat and polarised transition operators, write them to hopping_*.in / coulomb_*.in /
transop_*.in and Fock lists of up to ten million lines, call the Fortran solver, and read
pole files back to build their spectra (edrixs/iostream.py:279-323,
edrixs/plot_spectrum.py:9-61).  ``SiamSession`` takes those tensors directly, keeps the
Hamiltonians, Fock bases and ground states resident on the GPU between calls, and returns
what the callers return:

* ``ed``   -> (eval_i, denmat, v_noccu)               (ed_siam_fort with do_ed = 1)
* ``xas``  -> (xas (n_omega, n_pol), poles per pol)   (xas_siam_fort)
* ``rixs`` -> (rixs (n_omega, n_eloss, n_pol), poles[omega][pol])  (rixs_siam_fort)

Matrices are built from the nonzeros of emat / umat in the order write_emat / write_umat
emit them (edrixs/iostream.py:165-238), so the CSR equals the one the files give, up to the
15 decimals the text keeps.  Pole dicts carry unrounded coefficients (the files round them to
10 decimals, src/io.f90:532-537).  The physics that produces emat, umat and the transition
operators (Slater integrals, spin-orbit coupling, polarisation geometry) stays with the caller.
"""
import numpy as np
import torch

from . import device, fedrixs, rixs as rx, siam


def _terms(t):
    return siam.nonzero_terms(np.asarray(t, dtype=np.complex128))


def _gamma(g, n):
    g = np.asarray(g, dtype=np.float64)
    return np.full(n, float(g)) if g.ndim == 0 else g.astype(np.float64)


class SiamSession:
    """Resident state of one impurity problem: H_i over the v_noccu sector, H_n over the
    v_noccu + 1 sector with one core hole, and the ground states once ``ed`` has run.
    emat_*: (ntot, ntot) one-body matrices, umat_*: (ntot, ntot, ntot, ntot) Coulomb tensors,
    ntot = num_val_orbs + num_core_orbs, valence orbitals first (as the callers build them)."""

    def __init__(self, emat_i, umat_i, emat_n, umat_n, num_val_orbs, num_core_orbs, v_noccu):
        device.require_cuda()
        self.nv, self.nc, self.noccu = int(num_val_orbs), int(num_core_orbs), int(v_noccu)
        self.hop_i, self.coul_i = _terms(emat_i), _terms(umat_i)
        self.hop_n, self.coul_n = _terms(emat_n), _terms(umat_n)
        self.bi = device.fock_unrank(self.nv, self.noccu)
        self.bn = device.fock_unrank(self.nv, self.noccu + 1)
        self.Hi = device.build_csr(device.HAM_I, self.bi, self.hop_i, self.coul_i, num_val_orbs=self.nv)
        self._Hn = None
        self.gs_e = None
        self.gs_v = None

    @property
    def Hn(self):
        if self._Hn is None:
            self._Hn = device.build_csr(device.HAM_N, self.bn, self.hop_n, self.coul_n, num_val_orbs=self.nv,
                                        num_core_orbs=self.nc)
        return self._Hn

    def ed(self, *, ed_solver=2, neval=1, nvector=1, maxiter=1000, eigval_tol=1e-8, min_ndim=1000):
        """Lowest eigenpairs of H_i (src/ed_driver.f90:65-181 with these config.in values) and
        the density matrix of each of the nvector eigenvectors, denmat[k, i, j] = <c+_i c_j>
        (src/ed_driver.f90:194-248).  The eigenvectors stay resident for xas / rixs."""
        cfg = dict(ed_solver=ed_solver, neval=neval, nvector=nvector, maxiter=maxiter, eigval_tol=eigval_tol,
                   min_ndim=min_ndim)
        e, v = fedrixs.ed_core(cfg, self.Hi)
        self.gs_e, self.gs_v = np.asarray(e, dtype=np.float64), v.contiguous()
        dm = device.denmat(self.bi, self.nv, self.gs_v).cpu().numpy() if v.shape[1] else None
        return self.gs_e.copy(), dm, self.noccu

    def _ground(self, num_gs):
        if self.gs_v is None or self.gs_v.shape[1] < num_gs:
            raise ValueError(f"SiamSession: run ed(nvector >= {num_gs}) first")
        return self.gs_e[:num_gs], self.gs_v[:, :num_gs].contiguous()

    def _pole_dict(self, alpha, beta, norm, neff, e0):
        """read_poles_from_file's dict (edrixs/iostream.py:279-323) for a set of Lanczos runs."""
        ne = [int(x) for x in neff]
        return {"npoles": ne, "eigval": [float(x) for x in e0], "norm": [float(x) for x in norm],
                "alpha": [alpha[i, :n].tolist() for i, n in enumerate(ne)],
                "beta": [beta[i, :n].tolist() for i, n in enumerate(ne)]}

    def xas(self, ominc, trans, *, gamma_c=0.1, num_gs=1, nkryl=200, temperature=1.0):
        """XAS as xas_siam_fort returns it.  trans: one entry per polarisation, each a (ntot,
        ntot) transition matrix (the matrix the caller writes to transop_xas.in), or a list of
        matrices whose spectra are averaged (the caller's 'isotropic' entry).  Per ground state
        the Krylov space of D|g> on H_n (src/xas_driver.f90, src/lanczos.f90:210-303); all
        ground states and components of an entry run as one block."""
        ominc = np.asarray(ominc, dtype=np.float64)
        gam = _gamma(gamma_c, len(ominc))
        gs_e, gs_v = self._ground(num_gs)
        w = rx.boltz(gs_e, temperature)
        xas = np.zeros((len(ominc), len(trans)))
        poles = []
        for it, entry in enumerate(trans):
            mats = entry if isinstance(entry, (list, tuple)) else [entry]
            phis = []
            for T in mats:
                D = device.build_csr(device.TRANS_I, self.bn, _terms(T), right=self.bi, num_val_orbs=self.nv,
                                     num_core_orbs=self.nc)
                phis.append(device.spmm(D, gs_v))
            kr = device.krylov(self.Hn, torch.cat(phis, dim=1).contiguous(), int(nkryl))
            al, be, nrm, ne = (kr.alpha.cpu().numpy(), kr.beta.cpu().numpy(), kr.norm.cpu().numpy(),
                               kr.neff.cpu().numpy())
            dicts = []
            for c in range(len(mats)):
                sl = slice(c * num_gs, (c + 1) * num_gs)
                dicts.append(self._pole_dict(al[sl], be[sl], nrm[sl], ne[sl], gs_e))
                sp = device.cf_spectrum(kr.neff[sl], kr.alpha[sl], kr.beta[sl], gs_e, nrm[sl], w, ominc, gam)
                xas[:, it] += sp.cpu().numpy()
            xas[:, it] /= len(mats)
            poles.append(dicts[0] if len(mats) == 1 else dicts)
        return xas, poles

    def rixs(self, ominc, eloss, pairs, *, gamma_c=0.1, gamma_f=0.1, num_gs=1, nkryl=200, linsys_max=1000,
             linsys_tol=1e-10, temperature=1.0):
        """RIXS as rixs_siam_fort returns it.  pairs: one (trans_i, trans_f) per polarisation
        pair -- trans_i the absorption operator the caller writes to transop_rixs_i.in, trans_f
        the emission operator whose conjugate transpose it writes to transop_rixs_f.in.  All
        incident energies, pairs and ground states are one batched solve (rixs.rixs_spectra:
        the shifted MINRES systems of src/linsys.f90:3-128 share Krylov spaces, then one block
        Lanczos on H_f = H_i)."""
        ominc = np.asarray(ominc, dtype=np.float64)
        eloss = np.asarray(eloss, dtype=np.float64)
        gs_e, gs_v = self._ground(num_gs)
        ins, outs, idx = [], [], []
        for ti, tf in pairs:
            ti, tf = np.asarray(ti, dtype=np.complex128), np.asarray(tf, dtype=np.complex128)
            a = next((q for q, x in enumerate(ins) if np.array_equal(x, ti)), None)
            if a is None:
                ins.append(ti)
                a = len(ins) - 1
            b = next((q for q, x in enumerate(outs) if np.array_equal(x, tf)), None)
            if b is None:
                outs.append(tf)
                b = len(outs) - 1
            idx.append((a, b))
        Din = [device.build_csr(device.TRANS_I, self.bn, _terms(T), right=self.bi, num_val_orbs=self.nv,
                                num_core_orbs=self.nc) for T in ins]
        Dout = [device.build_csr(device.TRANS_F, self.bi, _terms(np.conj(T).T), right=self.bn,
                                 num_val_orbs=self.nv, num_core_orbs=self.nc) for T in outs]
        P = rx.RixsProblem(Hn=self.Hn, Hf=self.Hi, Din=Din, Dout=Dout, gs_e=gs_e, gs_v=gs_v)
        res = rx.rixs_spectra(P, ominc, _gamma(gamma_c, len(ominc)), eloss, _gamma(gamma_f, len(eloss)),
                              nkryl=int(nkryl), linsys_tol=linsys_tol, linsys_max=int(linsys_max),
                              temperature=temperature)
        npin, npout, n_om = len(Din), len(Dout), len(ominc)
        out = np.stack([res.spectra[:, :, a * npout + b] for a, b in idx], axis=-1)
        pl = res.poles
        al, be, nrm, ne = (pl["alpha"].cpu().numpy(), pl["beta"].cpu().numpy(), pl["norm"].cpu().numpy(),
                           pl["neff"].cpu().numpy())
        poles = []
        for w_ in range(n_om):
            per = []
            for a, b in idx:
                cols = [((b * npin + a) * num_gs + g) * n_om + w_ for g in range(num_gs)]
                per.append(self._pole_dict(al[cols], be[cols], nrm[cols], ne[cols], gs_e))
            poles.append(per)
        return out, poles
