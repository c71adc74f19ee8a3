"""The file family of the reference's two-valence-shell callers (ed_2v1c_fort, xas_2v1c_fort,
rixs_2v1c_fort, edrixs/solvers.py:718-1818) through the oracle.

tests/golden/callers_2v1c holds the files those callers write for t2g + p valence shells and
an s core (12 valence and 2 core orbitals, 10 valence electrons), including a quadrupolar
t2g <- s operator, and the dense matrices that the reference's manybody_operator.two_fermion
/ four_fermion build from the same terms.  The oracle's CSR builds must equal those matrices,
and its XAS and RIXS drivers must give the Kramers-Heisenberg spectra of those matrices
(the Lanczos runs reach the full dimension here, so the continued fractions are exact)."""
import os
import shutil

import numpy as np
import pytest

from edrixs_b200 import io as edxio
from oracle import drivers as odrv
from oracle import pyoracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden", "callers_2v1c")
NV, NC = 12, 2


@pytest.fixture(scope="module")
def dense():
    with np.load(os.path.join(G, "dense.npz")) as z:
        d = {k: z[k] for k in z.files}
    out = {}
    for key in d:
        if key.endswith("_shape"):
            name = key[:-6]
            M = np.zeros(tuple(d[key]), dtype=complex)
            M[d[name + "_row"], d[name + "_col"]] = d[name + "_val"]
            out[name] = M
    return out


def _files(name):
    d = {}
    for src in (os.path.join(G, "ed_00"), os.path.join(G, name)):
        for fn in os.listdir(src):
            d[fn] = os.path.join(src, fn)
    return d


def _close(A, B):
    assert A.shape == B.shape
    assert np.abs(A - B).max() <= 1e-13 * max(1.0, np.abs(B).max())


def test_2v1c_files_parse():
    cfg = edxio.read_config(os.path.join(G, "ed_00", "config.in"))
    assert cfg["num_val_orbs"] == NV and cfg["num_core_orbs"] == NC
    for name in ("xas_01", "xas_02", "rixs_03", "rixs_04"):
        f = _files(name)
        cfg = edxio.read_config(f["config.in"])
        assert cfg["num_val_orbs"] == NV and cfg["num_core_orbs"] == NC
        assert len(edxio.read_fock(f["fock_i.in"])) == 66 and len(edxio.read_fock(f["fock_n.in"])) == 12
        for fn in f:
            if fn.startswith("transop"):
                idx, val = edxio.read_hopping(f[fn])
                assert idx.min() >= 1 and idx.max() <= NV + NC and len(val) > 0


def test_2v1c_csr_equals_reference_operators(dense):
    f = _files("xas_01")
    fi, fn = orc.read_fock(f["fock_i.in"]), orc.read_fock(f["fock_n.in"])
    H = orc.build_csr("ham_i", fi, orc.read_terms(f["hopping_i.in"], 2), orc.read_terms(f["coulomb_i.in"], 4),
                      num_val_orbs=NV)
    _close(H.dense(), dense["H_i"])
    Hn = orc.build_csr("ham_n", fn, orc.read_terms(f["hopping_n.in"], 2), orc.read_terms(f["coulomb_n.in"], 4),
                       num_val_orbs=NV, num_core_orbs=NC)
    _close(Hn.dense(), dense["H_n"])
    for name in ("xas_01", "xas_02"):
        D = orc.build_csr("trans_i", fn, orc.read_terms(_files(name)["transop_xas.in"], 2), fock_right=fi,
                          num_val_orbs=NV, num_core_orbs=NC)
        _close(D.dense(), dense[f"D_{name}"])
    for name in ("rixs_03", "rixs_04"):
        g = _files(name)
        ff = orc.read_fock(g["fock_f.in"])
        Din = orc.build_csr("trans_i", fn, orc.read_terms(g["transop_rixs_i.in"], 2), fock_right=fi,
                            num_val_orbs=NV, num_core_orbs=NC)
        Dout = orc.build_csr("trans_f", ff, orc.read_terms(g["transop_rixs_f.in"], 2), fock_right=fn,
                             num_val_orbs=NV, num_core_orbs=NC)
        _close(Din.dense(), dense[f"D_in_{name}"])
        _close(Dout.dense(), dense[f"D_out_{name}"])
    # the quadrupolar and the dipolar operator reach different intermediate states
    assert not np.allclose(np.abs(dense["D_xas_01"]), np.abs(dense["D_xas_02"]))


def _workdir(tmp_path, name, e0, g0):
    d = tmp_path / name
    d.mkdir()
    for fn, src in _files(name).items():
        shutil.copy(src, d / fn)
    edxio.write_eigvec(str(d / "eigvec.1"), e0, g0)
    return str(d)


def _resolvent_spectrum(H, phi, e0, omegas, gamma):
    """-1/pi Im <phi|(w + i gamma + E_g - H)^-1|phi>: what the continued fraction of
    get_spectra_from_poles approximates."""
    ev, U = np.linalg.eigh(H)
    w2 = np.abs(U.conj().T @ phi) ** 2
    z = omegas[:, None] + 1j * gamma + e0 - ev[None, :]
    return -np.imag((w2[None, :] / z).sum(axis=1)) / np.pi


def test_2v1c_xas_and_rixs_match_kramers_heisenberg(dense, tmp_path):
    e, v = np.linalg.eigh(dense["H_i"])
    assert e[1] - e[0] > 1e-3          # a non-degenerate ground state
    e0, g0 = float(e[0]), v[:, 0]
    edge = np.linalg.eigvalsh(dense["H_n"])[0] - e0
    om = edge + np.linspace(-3.0, 12.0, 301)
    for name in ("xas_01", "xas_02"):
        (a, b, nrm, neff, eg), = odrv.xas(_workdir(tmp_path, name, e0, g0))
        poles = {"npoles": [neff], "eigval": [eg], "norm": [nrm], "alpha": [a], "beta": [b]}
        spec = orc.spectra_from_poles(poles, om, 0.3, 1.0)
        exact = _resolvent_spectrum(dense["H_n"], dense[f"D_{name}"] @ g0, e0, om, 0.3)
        assert np.abs(spec - exact).max() <= 1e-10 * np.abs(exact).max()
    eloss = np.linspace(-0.5, 6.0, 131)
    for name in ("rixs_03", "rixs_04"):
        cfg = edxio.read_config(_files(name)["config.in"])
        (a, b, nrm, neff, eg, its), = odrv.rixs(_workdir(tmp_path, name, e0, g0))
        poles = {"npoles": [neff], "eigval": [eg], "norm": [nrm], "alpha": [a], "beta": [b]}
        spec = orc.spectra_from_poles(poles, eloss, 0.1, 1.0)
        z = cfg["omega_in"] + e0 + 1j * cfg["gamma_in"]
        x = np.linalg.solve(z * np.eye(len(dense["H_n"])) - dense["H_n"], dense[f"D_in_{name}"] @ g0)
        exact = _resolvent_spectrum(dense["H_i"], dense[f"D_out_{name}"] @ x, e0, eloss, 0.1)
        assert np.abs(spec - exact).max() <= 1e-9 * np.abs(exact).max()
