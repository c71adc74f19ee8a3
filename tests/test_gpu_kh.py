"""The drop-in solvers on the GPU against the reference's Kramers-Heisenberg spectra.

The files of tests/golden/kh_1v1c (written by the reference's ed_1v1c_fort /
xas_1v1c_fort / rixs_1v1c_fort for a d8 ion with a 2p core) go through ed_fsolver,
xas_fsolver and rixs_fsolver of edrixs_b200.fedrixs; the spectra from the pole files they
write must equal those of the reference's pure-Python solvers (xas_1v1c_py, rixs_1v1c_py)
within 1e-8 relative L-inf (Lanczos to the full dimension, MINRES to 1e-13)."""
import os
import shutil

import numpy as np
import pytest

from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
KH = os.path.join(HERE, "golden", "kh_1v1c")


def _spec(d, prefix, grid, gamma, T):
    from edrixs_b200 import io
    pd = io.read_poles([os.path.join(d, f"{prefix}.1")])
    return orc.spectra_from_poles(pd, grid, gamma, T)


def test_drop_in_matches_kramers_heisenberg(cuda, tmp_path, monkeypatch):
    from edrixs_b200 import fedrixs
    with np.load(os.path.join(KH, "kh_spectra.npz")) as z:
        g = {k: z[k] for k in z.files}
    T = float(g["temperature"])
    base = tmp_path / "ed"
    shutil.copytree(os.path.join(KH, "ed_00"), base)
    cfg = (base / "config.in").read_text().replace("idump=.false.", "idump=.true.")
    (base / "config.in").write_text(cfg)
    monkeypatch.chdir(base)
    fedrixs.ed_fsolver(0, 0, 1)
    e0 = float(np.loadtxt("eigvals.dat", ndmin=2)[0, 1])
    assert abs(e0 - g["eval_i"][0]) < 1e-10

    def run(name, solver):
        d = tmp_path / name
        shutil.copytree(base, d)
        for fn in os.listdir(os.path.join(KH, name)):
            shutil.copy(os.path.join(KH, name, fn), d / fn)
        monkeypatch.chdir(d)
        solver(0, 0, 1)
        return str(d)

    for ip, name in enumerate(["xas_01", "xas_02"]):
        d = run(name, fedrixs.xas_fsolver)
        s = _spec(d, "xas_poles", g["ominc"], float(g["gamma_c_xas"]), T)
        ref = g["xas"][:, ip]
        assert np.max(np.abs(s - ref)) / np.max(np.abs(ref)) < 1e-8
    names = sorted(n for n in os.listdir(KH) if n.startswith("rixs_"))
    npol = g["rixs"].shape[2]
    for k, name in enumerate(names):
        iw, ip = divmod(k, npol)
        d = run(name, fedrixs.rixs_fsolver)
        s = _spec(d, "rixs_poles", g["eloss"], float(g["gamma_f"]), T)
        ref = g["rixs"][iw, :, ip]
        assert np.max(np.abs(s - ref)) / np.max(np.abs(ref)) < 1e-8, name
