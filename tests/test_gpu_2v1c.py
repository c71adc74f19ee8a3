"""The drop-in solvers on the GPU with the files of the reference's two-valence-shell callers
(ed_2v1c_fort, xas_2v1c_fort, rixs_2v1c_fort, edrixs/solvers.py:718-1818): t2g + p valence
shells and an s core, including a quadrupolar t2g <- s transition operator.

ED: eigvals.dat against the dense eigenvalues of the reference's own manybody_operator
matrices (tests/golden/callers_2v1c/dense.npz).  XAS and RIXS: the spectra of the drop-in's
pole files (read back as the reference's callers read them) against the exact
Kramers-Heisenberg spectra of those matrices; the Lanczos runs reach the full dimension here,
so the continued fractions are exact up to the 10 decimals of the files."""
import os
import shutil

import numpy as np
import pytest

from edrixs_b200 import io as edxio
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden", "callers_2v1c")


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


def _stage(tmp_path, name, e0=None, g0=None):
    """A working directory with the ED files and those of one XAS / RIXS caller run."""
    d = tmp_path / (name + "_run")
    d.mkdir()
    for src in (os.path.join(G, "ed_00"), os.path.join(G, name)):
        for fn in os.listdir(src):
            shutil.copy(os.path.join(src, fn), d / fn)
    if g0 is not None:
        edxio.write_eigvec(str(d / "eigvec.1"), e0, g0)
    return d


def _kh(H, phi, e0, omegas, gamma):
    ev, U = np.linalg.eigh(H)
    w2 = np.abs(U.conj().T @ phi) ** 2
    z = omegas[:, None] + 1j * gamma + e0 - ev[None, :]
    return -np.imag((w2[None, :] / z).sum(axis=1)) / np.pi


def test_2v1c_ed_xas_rixs_on_the_gpu(cuda, dense, tmp_path, monkeypatch):
    from edrixs_b200 import fedrixs
    e, v = np.linalg.eigh(dense["H_i"])
    # ED on the caller's files: eigenvalues as the dense matrices have them
    d = tmp_path / "ed_00"
    shutil.copytree(os.path.join(G, "ed_00"), d)
    monkeypatch.chdir(d)
    fedrixs.ed_fsolver(0, 0, 1)
    _, ours = np.loadtxt("eigvals.dat", unpack=True, ndmin=2)
    assert np.abs(ours - e[:len(ours)]).max() < 1e-9
    e0, g0 = float(e[0]), v[:, 0]
    edge = np.linalg.eigvalsh(dense["H_n"])[0] - e0
    om = edge + np.linspace(-3.0, 12.0, 301)
    for name in ("xas_01", "xas_02"):
        monkeypatch.chdir(_stage(tmp_path, name, e0, g0))
        fedrixs.xas_fsolver(0, 0, 1)
        spec = orc.spectra_from_poles(edxio.read_poles(["xas_poles.1"]), om, 0.3, 1.0)
        exact = _kh(dense["H_n"], dense[f"D_{name}"] @ g0, e0, om, 0.3)
        assert np.abs(spec - exact).max() <= 1e-6 * np.abs(exact).max(), name
    eloss = np.linspace(-0.5, 6.0, 131)
    for name in ("rixs_03", "rixs_04"):
        monkeypatch.chdir(_stage(tmp_path, name, e0, g0))
        cfg = edxio.read_config("config.in")
        fedrixs.rixs_fsolver(0, 0, 1)
        poles = edxio.read_poles(["rixs_poles.1"])
        z = cfg["omega_in"] + e0 + 1j * cfg["gamma_in"]
        x = np.linalg.solve(z * np.eye(len(dense["H_n"])) - dense["H_n"], dense[f"D_in_{name}"] @ g0)
        phi = dense[f"D_out_{name}"] @ x
        nrm = float(np.vdot(phi, phi).real)
        # the file keeps the normalisation to 10 decimals; compare it there and the spectrum
        # with the normalisation divided out
        assert abs(poles["norm"][0] - nrm) <= 6e-11
        spec = orc.spectra_from_poles(poles, eloss, 0.1, 1.0) / poles["norm"][0]
        exact = _kh(dense["H_i"], phi, e0, eloss, 0.1) / nrm
        assert np.abs(spec - exact).max() <= 1e-6 * np.abs(exact).max(), name
