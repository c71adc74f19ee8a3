"""The oracle's XAS and RIXS drivers against an answer the reference computes another way.

tests/golden/kh_1v1c holds, for a d8 ion with a 2p core (45 initial, 60 intermediate
states): the XAS and RIXS spectra of the reference's pure-Python Kramers-Heisenberg solvers
(xas_1v1c_py / rixs_1v1c_py on the eigenstates of ed_1v1c_py, edrixs/solvers.py:28-571),
and the input files that its Fortran-path callers (ed_1v1c_fort, xas_1v1c_fort,
rixs_1v1c_fort) write for the same ion.  Lanczos to the full dimension and MINRES to 1e-13
reproduce the Kramers-Heisenberg sums, so the oracle drivers (xas_driver.f90,
rixs_driver.f90 restated) on those files must give the same spectra.  This pins the XAS and
RIXS paths of the oracle, which the reference's own tests leave unpinned."""
import os
import shutil

import numpy as np
import pytest

from oracle import drivers as odrv
from oracle import pyoracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
KH = os.path.join(HERE, "golden", "kh_1v1c")


def _workdir(tmp_path, name, gs):
    d = tmp_path / name
    d.mkdir()
    for src in (os.path.join(KH, "ed_00"), os.path.join(KH, name)):
        for fn in os.listdir(src):
            shutil.copy(os.path.join(src, fn), d / fn)
    from edrixs_b200 import io as edxio
    edxio.write_eigvec(str(d / "eigvec.1"), gs[0], gs[1])
    return str(d)


def _poles(runs):
    return {"npoles": [r[3] for r in runs], "eigval": [r[4] for r in runs], "norm": [r[2] for r in runs],
            "alpha": [r[0] for r in runs], "beta": [r[1] for r in runs]}


@pytest.fixture(scope="module")
def golden():
    with np.load(os.path.join(KH, "kh_spectra.npz")) as z:
        g = {k: z[k] for k in z.files}
    e, v, H, fock, cfg = odrv.ed(os.path.join(KH, "ed_00"))
    assert abs(e[0] - g["eval_i"][0]) < 1e-10
    assert g["eval_i"][1] - g["eval_i"][0] > 1e-3  # a non-degenerate ground state
    return g, (e[0], v[:, 0])


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_xas_matches_kramers_heisenberg(golden, tmp_path):
    g, gs = golden
    for ip, name in enumerate(["xas_01", "xas_02"]):
        runs = odrv.xas(_workdir(tmp_path, name, gs))
        spec = orc.spectra_from_poles(_poles(runs), g["ominc"], float(g["gamma_c_xas"]), float(g["temperature"]))
        assert rel(spec, g["xas"][:, ip]) < 1e-10


def test_rixs_matches_kramers_heisenberg(golden, tmp_path):
    g, gs = golden
    names = sorted(n for n in os.listdir(KH) if n.startswith("rixs_"))
    n_om, npol = len(g["ominc_rixs"]), g["rixs"].shape[2]
    assert len(names) == n_om * npol  # the caller runs the solver per incident energy and polarisation
    for k, name in enumerate(names):
        iw, ip = divmod(k, npol)
        runs = odrv.rixs(_workdir(tmp_path, name, gs))
        spec = orc.spectra_from_poles(_poles(runs), g["eloss"], float(g["gamma_f"]), float(g["temperature"]))
        assert rel(spec, g["rixs"][iw, :, ip]) < 1e-10, (name, rel(spec, g["rixs"][iw, :, ip]))


def test_spectra_of_both_hamiltonians_match_reference():
    """All 45 initial and 60 intermediate eigenvalues of the oracle's H_i and H_n, built from
    the files the reference's callers wrote, equal those of ed_1v1c_py (which builds both
    Hamiltonians with its own two_fermion / four_fermion and diagonalises them densely)."""
    with np.load(os.path.join(KH, "kh_spectra.npz")) as z:
        eval_i, eval_n = z["eval_i"], z["eval_n"]
    base, xd = os.path.join(KH, "ed_00"), os.path.join(KH, "xas_01")
    cfg = odrv._cfg(os.path.join(xd, "config.in"))
    nv, nc = cfg["num_val_orbs"], cfg["num_core_orbs"]
    Hi = orc.build_csr("ham_i", orc.read_fock(os.path.join(base, "fock_i.in")),
                       orc.read_terms(os.path.join(base, "hopping_i.in"), 2),
                       orc.read_terms(os.path.join(base, "coulomb_i.in"), 4), num_val_orbs=nv)
    Hn = orc.build_csr("ham_n", orc.read_fock(os.path.join(xd, "fock_n.in")),
                       orc.read_terms(os.path.join(base, "hopping_n.in"), 2),
                       orc.read_terms(os.path.join(base, "coulomb_n.in"), 4), num_val_orbs=nv, num_core_orbs=nc)
    assert Hi.nrows == len(eval_i) and Hn.nrows == len(eval_n)
    assert np.allclose(np.linalg.eigvalsh(Hi.dense()), eval_i, atol=1e-10)
    assert np.allclose(np.linalg.eigvalsh(Hn.dense()), eval_n, atol=1e-10)


def test_thermal_xas_rixs_match_kramers_heisenberg(tmp_path):
    """Three ground states with Boltzmann weights at 3000 K (num_gs = 3: eigvec.1..3, one
    pole set each, summed by get_spectra_from_poles) against gs_list = [0, 1, 2] of the
    reference's Kramers-Heisenberg solvers."""
    from edrixs_b200 import io as edxio
    with np.load(os.path.join(KH, "kh_spectra.npz")) as z:
        g = {k: z[k] for k in z.files}
    base = os.path.join(KH, "ed_00")
    Hi = orc.build_csr("ham_i", orc.read_fock(os.path.join(base, "fock_i.in")),
                       orc.read_terms(os.path.join(base, "hopping_i.in"), 2),
                       orc.read_terms(os.path.join(base, "coulomb_i.in"), 4), num_val_orbs=10)
    e, v = np.linalg.eigh(Hi.dense())
    T = float(g["temperature_thermal"])

    def workdir(name):
        d = tmp_path / name
        d.mkdir()
        for src in (base, os.path.join(KH, name)):
            for fn in os.listdir(src):
                shutil.copy(os.path.join(src, fn), d / fn)
        for k in range(3):
            edxio.write_eigvec(str(d / f"eigvec.{k + 1}"), e[k], v[:, k])
        return str(d)

    runs = odrv.xas(workdir("xast_15"))
    assert len(runs) == 3
    spec = orc.spectra_from_poles(_poles(runs), g["ominc"], float(g["gamma_c_xas"]), T)
    assert rel(spec, g["xas_thermal"][:, 0]) < 1e-10
    for iw, name in enumerate(["rixst_16", "rixst_17"]):
        runs = odrv.rixs(workdir(name))
        spec = orc.spectra_from_poles(_poles(runs), g["eloss"], float(g["gamma_f"]), T)
        assert rel(spec, g["rixs_thermal"][iw, :, 0]) < 1e-10
