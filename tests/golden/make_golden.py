"""Generate the golden fixtures of tests/golden from the reference's own Python layer.

Run once where the reference is importable:
    python tests/golden/make_golden.py /path/to/edrixs-reference

What it writes (all small):
  known_answer/      the case of edrixs/tests/test_fortran.py:8-42 -- config.in,
                     hopping_i.in, coulomb_i.in, fock_i.in exactly as that test writes them,
                     plus expected_eigvals.txt from build_opers + scipy.linalg.eigh (:14-17).
  dense_small.npz    a 12-orbital SIAM (10 d + 2 bath, 2p core): the term lists as the files
                     carry them and the dense matrices of H_i, H_n, D_in, D_out built by the
                     reference's manybody_operator.two_fermion / four_fermion
                     (edrixs/manybody_operator.py:52-176) on bases ordered like the Fortran
                     rows (core-major intermediate index, src/ham.f90:424-446).
  fock_digests.json  sha256 of the sorted get_fock_full_N(norb, N) arrays (int64, little
                     endian) for the workload sizes, plus two explicit small lists.
  spectra.npz        random pole sets and get_spectra_from_poles (edrixs/plot_spectrum.py:9-61)
                     output on XAS/RIXS-like grids; boltz_dist (edrixs/utils.py:54-73) values.
  siam_callers/      the exact files ed_siam_fort (do_ed=2), xas_siam_fort and rixs_siam_fort
                     write before calling the solver (captured with a recording stand-in for
                     edrixs.fedrixs).
  denmat.npz         <c+_i c_j> of the two lowest eigenstates of the dense_small H_i, every
                     operator built by manybody_operator.two_fermion.
  kh_1v1c/           a d8 ion with a 2p core: XAS and RIXS spectra from the reference's
                     pure-Python Kramers-Heisenberg solvers (xas_1v1c_py, rixs_1v1c_py on
                     ed_1v1c_py eigenstates) and the input files its Fortran-path callers write
                     for the same ion; also a thermal case (3 ground states at 3000 K).
  callers_2v1c/      the files ed_2v1c_fort, xas_2v1c_fort (dipole and quadrupole) and
                     rixs_2v1c_fort write for t2g + p valence shells and an s core, and the dense
                     matrices two_fermion / four_fermion build from the same terms.
  search_gs/         the reference's ground-state search over N (ed_siam_fort, do_ed=0) for a
                     p shell with one bath site: its term files, the N of every solver call,
                     search_gs.log and search_result.dat (solver calls answered by the oracle).
"""
import hashlib
import json
import os
import shutil
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def import_reference(path):
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.path.insert(0, path)
    import edrixs
    return edrixs


class FakeComm:
    """The four calls solvers.py makes on an mpi4py communicator."""

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def py2f(self):
        return 0

    def Barrier(self):
        pass


def bits(state, norb):
    return np.array([(state >> p) & 1 for p in range(norb)], dtype=np.int64)


def known_answer(ed, out):
    os.makedirs(out, exist_ok=True)
    norb, noccu = 10, 2
    emat = ed.cf_cubic_d(1.5)
    umat = ed.get_umat_slater("d", 4.0, 2.0, 0.5)
    basis = ed.get_fock_bin_by_N(norb, noccu)
    H = ed.build_opers(2, emat, basis) + ed.build_opers(4, umat, basis)
    import scipy.linalg
    e, _ = scipy.linalg.eigh(H)
    cwd = os.getcwd()
    os.chdir(out)
    try:
        with open("config.in", "w") as f:
            f.write("&control\n"
                    "ed_solver     =   0\n"
                    "num_val_orbs  =   20\n"
                    "ncv           =   150\n"
                    f"neval         =   {len(e)}\n"
                    f"nvector       =   {len(e)}\n"
                    f"num_gs        =   {len(e)}\n"
                    "maxiter       =   1000\n"
                    "eigval_tol    =   1E-10\n"
                    "idump         =   .true.\n"
                    "&end\n")
        ed.write_fock_dec_by_N(norb, noccu)
        ed.write_emat(emat, "hopping_i.in")
        ed.write_umat(umat, "coulomb_i.in")
    finally:
        os.chdir(cwd)
    np.savetxt(os.path.join(out, "expected_eigvals.txt"), e, fmt="%.17e")


def dense_small(ed, out_path):
    from edrixs_b200 import siam
    nbath, N = 2, 3
    m = siam.make_siam(nbath, N, seed=7)
    nv, nc = m.nv, 6
    ntot = nv + nc
    # what the files carry (write_emat/write_umat text, parsed back)
    with tempfile.TemporaryDirectory() as td:
        paths = {}
        for name, t, fn in (("hop_i", m.emat_i, ed.write_emat), ("hop_n", m.emat_n, ed.write_emat),
                            ("coul_i", m.umat_i, ed.write_umat), ("coul_n", m.umat_n, ed.write_umat)):
            p = os.path.join(td, name)
            fn(t, p)
            paths[name] = p
        pol_in, pol_out = siam.rixs_polarisations()[1]
        t_in = siam.polarised_operator(m, pol_in)
        t_out_dag = np.conj(siam.polarised_operator(m, pol_out)).T
        ed.write_emat(t_in, os.path.join(td, "tr_i"))
        ed.write_emat(t_out_dag, os.path.join(td, "tr_f"))

        def load(p, nidx):
            with open(p) as f:
                n = int(f.readline().split()[0])
                rows = [f.readline().split() for _ in range(n)]
            idx = np.array([[int(r[k]) for k in range(nidx)] for r in rows], dtype=np.int32)
            val = np.array([float(r[nidx]) + 1j * float(r[nidx + 1]) for r in rows])
            return idx, val

        hi, ci = load(paths["hop_i"], 2), load(paths["coul_i"], 4)
        hn, cn = load(paths["hop_n"], 2), load(paths["coul_n"], 4)
        ti, tf = load(os.path.join(td, "tr_i"), 2), load(os.path.join(td, "tr_f"), 2)

    def tensor2(terms, n):
        t = np.zeros((n, n), dtype=complex)
        for (i, j), v in zip(terms[0], terms[1]):
            t[i - 1, j - 1] += v
        return t

    def tensor4(terms, n):
        t = np.zeros((n,) * 4, dtype=complex)
        for (i, j, k, l), v in zip(terms[0], terms[1]):
            t[i - 1, j - 1, k - 1, l - 1] += v
        return t

    fock_i = np.array(sorted(ed.get_fock_full_N(nv, N)), dtype=np.int64)
    fock_n = np.array(sorted(ed.get_fock_full_N(nv, N + 1)), dtype=np.int64)
    core_full = (1 << nc) - 1
    fock_core = [core_full - (1 << (nc - 1 - k)) for k in range(nc)]
    basis_i = [bits(s, nv) for s in fock_i]                                  # valence only
    basis_i_fullcore = [bits((core_full << nv) | s, ntot) for s in fock_i]   # with the core
    basis_n = [bits((fc << nv) | s, ntot) for fc in fock_core for s in fock_n]
    # H_i acts on valence-only states in build_ham_i: restrict the tensors to nv orbitals
    H_i = (ed.two_fermion(tensor2(hi, ntot)[:nv, :nv], basis_i) +
           ed.four_fermion(tensor4(ci, ntot)[:nv, :nv, :nv, :nv], basis_i))
    H_n = ed.two_fermion(tensor2(hn, ntot), basis_n) + ed.four_fermion(tensor4(cn, ntot), basis_n)
    D_in = ed.two_fermion(tensor2(ti, ntot), basis_n, basis_i_fullcore)
    D_out = ed.two_fermion(tensor2(tf, ntot), basis_i_fullcore, basis_n)

    def coo(Mx):
        r, c = np.nonzero(Mx)
        return r.astype(np.int32), c.astype(np.int32), Mx[r, c]

    data = dict(nv=nv, nc=nc, nelec=N, fock_i=fock_i, fock_n=fock_n,
                hop_i_idx=hi[0], hop_i_val=hi[1], coul_i_idx=ci[0], coul_i_val=ci[1],
                hop_n_idx=hn[0], hop_n_val=hn[1], coul_n_idx=cn[0], coul_n_val=cn[1],
                tr_i_idx=ti[0], tr_i_val=ti[1], tr_f_idx=tf[0], tr_f_val=tf[1])
    for name, Mx in (("H_i", H_i), ("H_n", H_n), ("D_in", D_in), ("D_out", D_out)):
        r, c, v = coo(Mx)
        data[f"{name}_row"], data[f"{name}_col"], data[f"{name}_val"] = r, c, v
        data[f"{name}_shape"] = np.array(Mx.shape)
    np.savez_compressed(out_path, **data)
    return {k: v.shape for k, v in data.items() if hasattr(v, "shape")}


def fock_digests(ed, out_path):
    res = {}
    for norb, N in ((20, 10), (20, 11), (24, 12), (26, 13)):
        a = np.array(sorted(ed.get_fock_full_N(norb, N)), dtype="<i8")
        res[f"{norb}_{N}"] = {"ndim": int(len(a)), "sha256": hashlib.sha256(a.tobytes()).hexdigest(),
                              "first": [int(x) for x in a[:3]], "last": [int(x) for x in a[-3:]]}
    res["explicit_4_2"] = [int(x) for x in sorted(ed.get_fock_full_N(4, 2))]
    res["explicit_6_3"] = [int(x) for x in sorted(ed.get_fock_full_N(6, 3))]
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)


def spectra(ed, out_path):
    rng = np.random.default_rng(11)
    poles = {"npoles": [], "eigval": [], "norm": [], "alpha": [], "beta": []}
    for g in range(3):
        neff = [40, 200, 1][g]
        poles["npoles"].append(neff)
        poles["eigval"].append(float(-12.3 + 0.01 * g))
        poles["norm"].append(float(rng.uniform(0.5, 2.0)))
        poles["alpha"].append(list(rng.uniform(-15, 5, neff)))
        poles["beta"].append(list(rng.uniform(0.1, 3.0, neff)))
    om_xas = np.linspace(-5, 15, 1000)
    om_rixs = np.linspace(-1, 12, 2000)
    gam_rixs = np.linspace(0.1, 0.4, 2000)
    s_xas = ed.get_spectra_from_poles(poles, om_xas, np.full(1000, 0.3), 300.0)
    s_rixs = ed.get_spectra_from_poles(poles, om_rixs, gam_rixs, 10.0)
    np.savez_compressed(out_path, npoles=np.array(poles["npoles"]), eigval=np.array(poles["eigval"]),
                        norm=np.array(poles["norm"]),
                        alpha=np.array([np.pad(a, (0, 200 - len(a))) for a in poles["alpha"]]),
                        beta=np.array([np.pad(b, (0, 200 - len(b))) for b in poles["beta"]]),
                        om_xas=om_xas, s_xas=s_xas, om_rixs=om_rixs, gam_rixs=gam_rixs, s_rixs=s_rixs,
                        boltz_e=np.array([-3.0, -2.99, -2.5]), boltz_T=np.array([1.0, 300.0, 3000.0]),
                        boltz=np.array([ed.boltz_dist([-3.0, -2.99, -2.5], T) for T in (1.0, 300.0, 3000.0)]))


def siam_callers(ed, out_dir):
    """Record what the reference's callers write for the solver (tiny model: 10 d + 2 bath)."""
    from edrixs_b200 import siam
    m = siam.make_siam(2, 3, seed=7)
    hopping = m.emat_i[:m.nv, :m.nv]
    slater = ([8.0, 10.0, 6.2], [8.0, 10.0, 6.2] + list(siam.DEFAULT_SLATER_VC))
    calls = {"n": 0}

    def recorder(kind):
        def fsolver(comm, my_id, num_procs):
            calls["n"] += 1
            d = os.path.join(out_dir, f"{kind}_{calls['n']}")
            os.makedirs(d, exist_ok=True)
            for fn in os.listdir("."):
                if fn.endswith(".in"):
                    shutil.copy(fn, os.path.join(d, fn))
            # minimal outputs so that the caller can go on
            if kind == "xas" or kind == "rixs":
                for g in range(1):
                    with open(f"{kind}_poles.{g + 1}", "w") as f:
                        f.write("#number_of_poles:            1\n#enegry:                  0.0\n"
                                "#normalization:           1.0\n    1      0.0      0.0\n")
        return fsolver

    mod = types.ModuleType("edrixs.fedrixs")
    mod.ed_fsolver = recorder("ed")
    mod.xas_fsolver = recorder("xas")
    mod.rixs_fsolver = recorder("rixs")
    sys.modules["edrixs.fedrixs"] = mod
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            comm = FakeComm()
            ed.ed_siam_fort(comm, ("d", "p"), 0, siam_type=1, v_noccu=3, hopping=m.emat_i[:10, :10],
                            slater=slater, c_soc=11.0, do_ed=2, ed_solver=2, neval=4, nvector=2, ncv=20,
                            idump=True, maxiter=1000, eigval_tol=1e-10, min_ndim=10)
            d = os.path.join(out_dir, "ed_do_ed2")
            os.makedirs(d, exist_ok=True)
            for fn in os.listdir("."):
                if fn.endswith(".in"):
                    shutil.copy(fn, os.path.join(d, fn))
            ed.xas_siam_fort(comm, ("d", "p"), 0, np.linspace(-2, 8, 11), gamma_c=0.3, v_noccu=3,
                             pol_type=[("linear", 0.0)], num_gs=1, nkryl=50, temperature=300.0)
            ed.rixs_siam_fort(comm, ("d", "p"), 0, np.array([1.5]), np.linspace(-0.5, 5, 11), gamma_c=0.6,
                              gamma_f=0.1, v_noccu=3, pol_type=[("linear", 0.0, "linear", np.pi / 2)],
                              num_gs=1, nkryl=50, linsys_max=500, linsys_tol=1e-10, temperature=300.0)
        finally:
            os.chdir(cwd)
    del hopping


def kh_1v1c(ed, out_dir):
    """An independent answer for the XAS and RIXS drivers: a d8 ion with a 2p core (45
    initial, 60 intermediate states), solved by the reference's pure-Python path --
    ed_1v1c_py (dense eigenproblems), xas_1v1c_py and rixs_1v1c_py (Kramers-Heisenberg sums
    over all eigenstates, edrixs/solvers.py:28-571) -- and the input files that the
    reference's Fortran-path callers ed_1v1c_fort / xas_1v1c_fort / rixs_1v1c_fort write for
    the same ion (captured with a recording stand-in for edrixs.fedrixs).  A Lanczos run to
    the full dimension reproduces the Kramers-Heisenberg spectra, so the oracle drivers on
    those files must give them."""
    rng = np.random.default_rng(17)
    a = rng.normal(scale=0.15, size=(10, 10)) + 1j * rng.normal(scale=0.15, size=(10, 10))
    cf = a + a.conj().T  # generic crystal field: a non-degenerate ground state
    kw = dict(shell_level=(0.0, -100.0), v_soc=(0.08, 0.1), c_soc=11.0, v_noccu=8,
              slater=([8.0, 10.0, 6.2], [8.0, 10.0, 6.2, 7.0, 6.0, 4.5, 2.6]), v_cfmat=cf)
    eval_i, eval_n, trans_op = ed.ed_1v1c_py(("d", "p"), **kw)
    edge = float(eval_n[0] - eval_i[0])
    ominc = edge + np.linspace(-2.0, 8.0, 41)
    eloss = np.linspace(-0.5, 6.0, 66)
    xas_pol = [("linear", 0.0), ("left", 0.0)]
    rixs_pol = [("linear", 0.0, "linear", np.pi / 2), ("linear", np.pi / 2, "linear", 0.0)]
    geo = dict(thin=0.6, phi=0.3)
    T = 10.0
    xas = ed.xas_1v1c_py(eval_i, eval_n, trans_op, ominc, gamma_c=0.3, pol_type=xas_pol, gs_list=[0],
                         temperature=T, **geo)
    rixs = ed.rixs_1v1c_py(eval_i, eval_n, trans_op, ominc[::8], eloss, gamma_c=0.6, gamma_f=0.1, thout=1.1,
                           pol_type=rixs_pol, gs_list=[0], temperature=T, **geo)
    # a thermal case: three ground states with Boltzmann weights at 3000 K
    Th = 3000.0
    xas_t = ed.xas_1v1c_py(eval_i, eval_n, trans_op, ominc, gamma_c=0.3, pol_type=xas_pol[:1], gs_list=[0, 1, 2],
                           temperature=Th, **geo)
    rixs_t = ed.rixs_1v1c_py(eval_i, eval_n, trans_op, ominc[8:17:8], eloss, gamma_c=0.6, gamma_f=0.1, thout=1.1,
                             pol_type=rixs_pol[:1], gs_list=[0, 1, 2], temperature=Th, **geo)
    calls = {"n": 0}

    def recorder(kind):
        def fsolver(comm, my_id, num_procs):
            calls["n"] += 1
            tag = "t" if "thermal" in calls else ""
            d = os.path.join(out_dir, f"{kind}{tag}_{calls['n']:02d}")
            os.makedirs(d, exist_ok=True)
            for fn in os.listdir("."):
                if fn.endswith(".in"):
                    shutil.copy(fn, os.path.join(d, fn))
            if kind in ("xas", "rixs"):  # minimal outputs so that the caller can go on
                import re
                ngs = int(re.search(r"num_gs=(\d+)", open("config.in").read()).group(1))
                for g in range(ngs):
                    with open(f"{kind}_poles.{g + 1}", "w") as f:
                        f.write("#number_of_poles:            1\n#enegry:                  0.0\n"
                                "#normalization:           1.0\n    1      0.0      0.0\n")
        return fsolver

    mod = types.ModuleType("edrixs.fedrixs")
    mod.ed_fsolver, mod.xas_fsolver, mod.rixs_fsolver = recorder("ed"), recorder("xas"), recorder("rixs")
    sys.modules["edrixs.fedrixs"] = mod
    if os.path.isdir(out_dir):
        shutil.rmtree(out_dir)
    os.makedirs(out_dir)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            comm = FakeComm()
            ed.ed_1v1c_fort(comm, ("d", "p"), do_ed=False, ed_solver=0, neval=3, nvector=1, min_ndim=1000, **kw)
            d = os.path.join(out_dir, "ed_00")  # do_ed=False: the files only, no solver call
            os.makedirs(d)
            for fn in os.listdir("."):
                if fn.endswith(".in"):
                    shutil.copy(fn, os.path.join(d, fn))
            ed.xas_1v1c_fort(comm, ("d", "p"), ominc, gamma_c=0.3, v_noccu=8, pol_type=xas_pol, num_gs=1,
                             nkryl=200, temperature=T, **geo)
            ed.rixs_1v1c_fort(comm, ("d", "p"), ominc[::8], eloss, gamma_c=0.6, gamma_f=0.1, v_noccu=8, thout=1.1,
                              pol_type=rixs_pol, num_gs=1, nkryl=200, linsys_max=1000, linsys_tol=1e-13,
                              temperature=T, **geo)
            calls["thermal"] = calls["n"]  # calls after this one are the thermal case
            ed.xas_1v1c_fort(comm, ("d", "p"), ominc, gamma_c=0.3, v_noccu=8, pol_type=xas_pol[:1], num_gs=3,
                             nkryl=200, temperature=Th, **geo)
            ed.rixs_1v1c_fort(comm, ("d", "p"), ominc[8:17:8], eloss, gamma_c=0.6, gamma_f=0.1, v_noccu=8,
                              thout=1.1, pol_type=rixs_pol[:1], num_gs=3, nkryl=200, linsys_max=1000,
                              linsys_tol=1e-13, temperature=Th, **geo)
        finally:
            os.chdir(cwd)
    # keep one copy of the files every call shares (Hamiltonian terms, initial basis)
    base = os.path.join(out_dir, "ed_00")
    for d in sorted(os.listdir(out_dir)):
        if d == "ed_00":
            continue
        for fn in os.listdir(os.path.join(out_dir, d)):
            p = os.path.join(out_dir, d, fn)
            q = os.path.join(base, fn)
            if os.path.exists(q) and open(p, "rb").read() == open(q, "rb").read():
                os.remove(p)
    np.savez(os.path.join(out_dir, "kh_spectra.npz"), eval_i=eval_i, eval_n=eval_n, ominc=ominc,
             ominc_rixs=ominc[::8], eloss=eloss, xas=xas, rixs=rixs, gamma_c_xas=0.3, gamma_c_rixs=0.6,
             gamma_f=0.1, temperature=T, xas_thermal=xas_t, rixs_thermal=rixs_t, ominc_rixs_thermal=ominc[8:17:8],
             temperature_thermal=Th)
    return sorted(os.listdir(out_dir))


def denmat_golden(ed, dense_path, out_path):
    """<c+_i c_j> of the ground state and of the first excited state of the dense_small H_i,
    each operator built by the reference's manybody_operator.two_fermion on the same basis
    (an independent route to what src/ed_driver.f90:194-248 computes)."""
    with np.load(dense_path) as z:
        d = {k: z[k] for k in z.files}
    nv = int(d["nv"])
    n = int(d["H_i_shape"][0])
    H = np.zeros((n, n), dtype=complex)
    H[d["H_i_row"], d["H_i_col"]] = d["H_i_val"]
    e, v = np.linalg.eigh(H)
    basis = [bits(int(st), nv) for st in d["fock_i"]]
    rho = np.zeros((2, nv, nv), dtype=complex)
    for i in range(nv):
        for j in range(nv):
            E = np.zeros((nv, nv), dtype=complex)
            E[i, j] = 1.0
            M = ed.two_fermion(E, basis)
            for k in range(2):
                rho[k, i, j] = v[:, k].conj() @ M @ v[:, k]
    np.savez(out_path, eigvals=e[:3], rho=rho)
    return float(e[1] - e[0]), float(e[2] - e[1])


def callers_2v1c(ed, out_dir):
    """Two valence shells and one core shell: t2g (6) + p (6) valence orbitals, an s core (2),
    10 valence electrons (66 initial, 2 x 12 intermediate states).  The files that
    ed_2v1c_fort (do_ed=False), xas_2v1c_fort (a p<-s dipole and a t2g<-s quadrupole
    operator) and rixs_2v1c_fort write, captured with a recording stand-in for
    edrixs.fedrixs, and the dense matrices the reference's manybody_operator.two_fermion /
    four_fermion build from the same terms (H_i, H_n, each transition operator), on bases
    ordered like the Fortran rows (core-major intermediate index, src/ham.f90:424-446)."""
    rng = np.random.default_rng(23)
    a = rng.normal(scale=0.2, size=(6, 6)) + 1j * rng.normal(scale=0.2, size=(6, 6))
    hv = rng.normal(scale=0.3, size=(6, 6)) + 1j * rng.normal(scale=0.3, size=(6, 6))
    shells = ("t2g", "p", "s")
    kw = dict(shell_level=(0.0, 2.0, -40.0), v1_soc=(0.05, 0.06), v2_soc=(0.02, 0.03), v_tot_noccu=10,
              slater=([4.0, 3.0, 2.0, 2.0, 1.0, 0.8, 0.5, 1.5, 1.0],
                      [4.0, 3.0, 2.0, 2.0, 1.0, 0.8, 0.5, 1.5, 1.0, 2.0, 0.7, 1.8, 0.6]),
              v1_cfmat=a + a.conj().T, hopping_v1v2=hv)
    calls = {"n": 0}

    def recorder(kind):
        def fsolver(comm, my_id, num_procs):
            calls["n"] += 1
            d = os.path.join(out_dir, f"{kind}_{calls['n']:02d}")
            os.makedirs(d, exist_ok=True)
            for fn in os.listdir("."):
                if fn.endswith(".in"):
                    shutil.copy(fn, os.path.join(d, fn))
            with open(f"{kind}_poles.1", "w") as f:
                f.write("#number_of_poles:            1\n#enegry:                  0.0\n"
                        "#normalization:           1.0\n    1      0.0      0.0\n")
        return fsolver

    mod = types.ModuleType("edrixs.fedrixs")
    mod.ed_fsolver, mod.xas_fsolver, mod.rixs_fsolver = recorder("ed"), recorder("xas"), recorder("rixs")
    sys.modules["edrixs.fedrixs"] = mod
    if os.path.isdir(out_dir):
        shutil.rmtree(out_dir)
    os.makedirs(out_dir)
    cwd = os.getcwd()
    geo = dict(thin=0.5, phi=0.2)
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            comm = FakeComm()
            ed.ed_2v1c_fort(comm, shells, do_ed=False, ed_solver=0, neval=2, nvector=1, min_ndim=1000, **kw)
            d = os.path.join(out_dir, "ed_00")
            os.makedirs(d)
            for fn in os.listdir("."):
                if fn.endswith(".in"):
                    shutil.copy(fn, os.path.join(d, fn))
            om = np.linspace(-2.0, 8.0, 5)
            ed.xas_2v1c_fort(comm, shells, om, gamma_c=0.3, v_tot_noccu=10, trans_to_which=2,
                             pol_type=[("linear", 0.0)], num_gs=1, nkryl=100, **geo)
            ed.xas_2v1c_fort(comm, shells, om, gamma_c=0.3, v_tot_noccu=10, trans_to_which=1,
                             pol_type=[("linear", 0.3)], num_gs=1, nkryl=100, **geo)
            # incident energies near the edge, where the RIXS amplitudes are large
            from oracle import pyoracle as orc
            e_i = np.linalg.eigvalsh(orc.build_csr(
                "ham_i", orc.read_fock("fock_i.in"), orc.read_terms("hopping_i.in", 2),
                orc.read_terms("coulomb_i.in", 4), num_val_orbs=12).dense())[0]
            e_n = np.linalg.eigvalsh(orc.build_csr(
                "ham_n", orc.read_fock("fock_n.in"), orc.read_terms("hopping_n.in", 2),
                orc.read_terms("coulomb_n.in", 4), num_val_orbs=12, num_core_orbs=2).dense())[0]
            ominc = round(float(e_n - e_i), 4) + np.array([0.5, 2.0])
            ed.rixs_2v1c_fort(comm, shells, ominc, np.linspace(-0.5, 4.0, 5), gamma_c=0.5,
                              gamma_f=0.1, v_tot_noccu=10, trans_to_which=2, thout=1.0,
                              pol_type=[("linear", 0.0, "linear", np.pi / 2)], num_gs=1, nkryl=100,
                              linsys_max=500, linsys_tol=1e-12, **geo)
        finally:
            os.chdir(cwd)
    base = os.path.join(out_dir, "ed_00")
    for d in sorted(os.listdir(out_dir)):
        if d == "ed_00":
            continue
        for fn in os.listdir(os.path.join(out_dir, d)):
            p = os.path.join(out_dir, d, fn)
            q = os.path.join(base, fn)
            stale = d.startswith("rixs") and fn == "transop_xas.in"   # left by the XAS calls
            if stale or (os.path.exists(q) and open(p, "rb").read() == open(q, "rb").read()):
                os.remove(p)

    # dense matrices from the reference's operator builders on the recorded terms
    def terms(path, nidx):
        with open(path) as f:
            n = int(f.readline().split()[0])
            rows = [f.readline().split() for _ in range(n)]
        return ([[int(r[k]) for k in range(nidx)] for r in rows],
                [float(r[nidx]) + 1j * float(r[nidx + 1]) for r in rows])

    def tensor(tm, n, nidx):
        t = np.zeros((n,) * nidx, dtype=complex)
        for idx, v in zip(*tm):
            t[tuple(i - 1 for i in idx)] += v
        return t

    nv, nc, N = 12, 2, 10
    ntot = nv + nc
    fock_i = np.array(sorted(ed.get_fock_full_N(nv, N)), dtype=np.int64)
    fock_n = np.array(sorted(ed.get_fock_full_N(nv, N + 1)), dtype=np.int64)
    core_full = (1 << nc) - 1
    fock_core = [core_full - (1 << (nc - 1 - k)) for k in range(nc)]
    basis_i = [bits(s, nv) for s in fock_i]
    basis_i_fullcore = [bits((core_full << nv) | s, ntot) for s in fock_i]
    basis_n = [bits((fc << nv) | s, ntot) for fc in fock_core for s in fock_n]
    ed0 = os.path.join(out_dir, "ed_00")
    H_i = (ed.two_fermion(tensor(terms(os.path.join(ed0, "hopping_i.in"), 2), ntot, 2)[:nv, :nv], basis_i) +
           ed.four_fermion(tensor(terms(os.path.join(ed0, "coulomb_i.in"), 4), ntot, 4)[:nv, :nv, :nv, :nv],
                           basis_i))
    H_n = (ed.two_fermion(tensor(terms(os.path.join(ed0, "hopping_n.in"), 2), ntot, 2), basis_n) +
           ed.four_fermion(tensor(terms(os.path.join(ed0, "coulomb_n.in"), 4), ntot, 4), basis_n))
    mats = {"H_i": H_i, "H_n": H_n}
    for d in sorted(os.listdir(out_dir)):
        for fn, rows, cols, name in (("transop_xas.in", basis_n, basis_i_fullcore, "D"),
                                     ("transop_rixs_i.in", basis_n, basis_i_fullcore, "D_in"),
                                     ("transop_rixs_f.in", basis_i_fullcore, basis_n, "D_out")):
            p = os.path.join(out_dir, d, fn)
            if os.path.exists(p):
                mats[f"{name}_{d}"] = ed.two_fermion(tensor(terms(p, 2), ntot, 2), rows, cols)
    data = {}
    for name, M in mats.items():
        r, c = np.nonzero(M)
        data[f"{name}_row"], data[f"{name}_col"] = r.astype(np.int32), c.astype(np.int32)
        data[f"{name}_val"], data[f"{name}_shape"] = M[r, c], np.array(M.shape)
    np.savez_compressed(os.path.join(out_dir, "dense.npz"), **data)
    return sorted(os.listdir(out_dir)), sorted(mats)


def search_gs(ed, out_dir, level=-6.0):
    """The reference's ground-state search over N (ed_siam_fort with do_ed=0,
    edrixs/solvers.py:2156-2263) on a p shell with one bath site (6 + 6 orbitals, N = 0..12,
    at most 924 states), general hybridisation (siam_type=1). Its
    ed_fsolver calls go to a stand-in that solves with the oracle (dense) and writes
    eigvals.dat / denmat.dat in the reference's formats; the reference's own loop reads them
    back, walks N, and writes search_gs.log and search_result.dat.  Kept: hopping_i.in and
    coulomb_i.in of the first call, the N of every call, both result files, and config.in of
    the last call (the one at the ground-state occupancy)."""
    from edrixs_b200 import io as edxio
    from oracle import pyoracle as orc
    rng = np.random.default_rng(5)
    a = rng.normal(0.0, 0.3, (6, 6)) + 1j * rng.normal(0.0, 0.3, (6, 6))
    hopping = np.zeros((12, 12), dtype=np.complex128)
    hopping[:6, :6] = (a + a.conj().T) / 2 + level * np.eye(6)
    hopping[6:, 6:] = np.diag(rng.uniform(-2.0, 2.0, 6))
    hopping[:6, 6:] = rng.normal(0.0, 0.6, (6, 6)) + 1j * rng.normal(0.0, 0.6, (6, 6))
    hopping[6:, :6] = hopping[:6, 6:].conj().T
    calls = []

    def ed_fsolver(comm, my_id, num_procs):
        cfg = edxio.read_config("config.in")
        fock = orc.read_fock("fock_i.in")
        if not calls:
            os.makedirs(out_dir, exist_ok=True)
            for fn in ("hopping_i.in", "coulomb_i.in"):
                shutil.copy(fn, os.path.join(out_dir, fn))
        calls.append(bin(int(fock[0])).count("1"))
        nv = cfg["num_val_orbs"]
        H = orc.build_csr("ham_i", fock, orc.read_terms("hopping_i.in", 2), orc.read_terms("coulomb_i.in", 4),
                          num_val_orbs=nv)
        e, v = np.linalg.eigh(H.dense())
        nvec = min(cfg["nvector"], len(fock))
        edxio.write_eigvals("eigvals.dat", e[:min(cfg["neval"], len(fock))])
        edxio.write_denmat("denmat.dat", np.stack([orc.denmat(fock, nv, v[:, k]) for k in range(nvec)]))
        shutil.copy("config.in", os.path.join(out_dir, "config_last.in"))

    mod = types.ModuleType("edrixs.fedrixs")
    mod.ed_fsolver = ed_fsolver
    sys.modules["edrixs.fedrixs"] = mod
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            eval_i, denmat, noccu = ed.ed_siam_fort(FakeComm(), ("p", "s"), 1, siam_type=1, hopping=hopping,
                                                   slater=([4.0, 3.0], [4.0, 3.0]), do_ed=0,
                                                   ed_solver=2, neval=2, nvector=1, min_ndim=10)
            for fn in ("search_gs.log", "search_result.dat"):
                shutil.copy(fn, os.path.join(out_dir, fn))
        finally:
            os.chdir(cwd)
    with open(os.path.join(out_dir, "calls.json"), "w") as f:
        json.dump({"n_per_call": calls, "noccu_gs": int(noccu), "eval_i": [float(x) for x in eval_i]}, f)
    return calls, int(noccu)


def main(ref):
    ed = import_reference(ref)
    known_answer(ed, os.path.join(HERE, "known_answer"))
    print("dense_small", dense_small(ed, os.path.join(HERE, "dense_small.npz")))
    fock_digests(ed, os.path.join(HERE, "fock_digests.json"))
    spectra(ed, os.path.join(HERE, "spectra.npz"))
    siam_callers(ed, os.path.join(HERE, "siam_callers"))
    print("kh_1v1c", kh_1v1c(ed, os.path.join(HERE, "kh_1v1c")))
    print("denmat", denmat_golden(ed, os.path.join(HERE, "dense_small.npz"), os.path.join(HERE, "denmat.npz")))
    print("callers_2v1c", callers_2v1c(ed, os.path.join(HERE, "callers_2v1c")))
    print("search_gs", search_gs(ed, os.path.join(HERE, "search_gs")))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
