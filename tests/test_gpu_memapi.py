"""The in-memory SIAM API (edrixs_b200/memapi.py) against the file-based drop-in, on the files
the reference's own ed_siam_fort / xas_siam_fort / rixs_siam_fort wrote (tests/golden/
siam_callers).  The tensors are read back from those files, passed in memory, and the
results (eigenvalues, spectra, Lanczos coefficients) must equal what the drop-in solvers
produce from the files: spectra within 1e-6 relative L-inf, coefficients within the 1e-10
rounding of the pole files (src/io.f90:532-537)."""
import os
import shutil

import numpy as np
import pytest

from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu

NTOT, NV, NC = 16, 10, 6


def _dense(path, nidx):
    from edrixs_b200 import io
    idx, val = (io.read_coulomb if nidx == 4 else io.read_hopping)(path)
    t = np.zeros((NTOT,) * nidx, dtype=np.complex128)
    for ix, v in zip(np.asarray(idx).reshape(-1, nidx), np.asarray(val)):
        t[tuple(int(i) - 1 for i in ix)] += v
    return t


@pytest.fixture
def workdir(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    return tmp_path


def _session(src):
    from edrixs_b200 import io, memapi
    d = os.path.join(src, "ed_do_ed2")
    fock = io.read_fock(os.path.join(d, "fock_i.in"))
    noccu = bin(int(fock[0])).count("1")
    S = memapi.SiamSession(_dense(os.path.join(d, "hopping_i.in"), 2), _dense(os.path.join(d, "coulomb_i.in"), 4),
                           _dense(os.path.join(d, "hopping_n.in"), 2), _dense(os.path.join(d, "coulomb_n.in"), 4),
                           NV, NC, noccu)
    e, dm, n = S.ed(ed_solver=2, neval=4, nvector=2, maxiter=1000, eigval_tol=1e-10, min_ndim=10)
    return S, e, dm, n


def _drop_in(src, workdir, kind):
    from edrixs_b200 import fedrixs
    for f in os.listdir(os.path.join(src, "ed_do_ed2")):
        shutil.copy(os.path.join(src, "ed_do_ed2", f), workdir)
    fedrixs.ed_fsolver(0, 0, 1)
    sub = [x for x in os.listdir(src) if x.startswith(kind)][0]
    for f in os.listdir(os.path.join(src, sub)):
        shutil.copy(os.path.join(src, sub, f), workdir)
    return os.path.join(src, sub)


def test_ed_and_xas_in_memory_equal_the_files(cuda, golden_dir, workdir):
    from edrixs_b200 import fedrixs, io
    src = os.path.join(golden_dir, "siam_callers")
    S, e, dm, noccu = _session(src)
    d = _drop_in(src, workdir, "xas")
    _, e_file = np.loadtxt("eigvals.dat", unpack=True)
    assert np.abs(e - e_file).max() < 1e-9
    dmf = np.loadtxt("denmat.dat")
    assert np.abs(dm[0].ravel() - (dmf[:NV * NV, 3] + 1j * dmf[:NV * NV, 4]).reshape(NV, NV).ravel()).max() < 1e-9
    fedrixs.xas_fsolver(0, 0, 1)
    poles_f = io.read_poles(["xas_poles.1"])
    ominc = np.linspace(-5.0, 15.0, 400)
    spec_f = orc.spectra_from_poles(poles_f, ominc, np.full(len(ominc), 0.3), 1.0)
    T = _dense(os.path.join(d, "transop_xas.in"), 2)
    xas, poles = S.xas(ominc, [T, [T, T]], gamma_c=0.3, num_gs=1, nkryl=50, temperature=1.0)
    assert xas.shape == (400, 2)
    for col in (0, 1):  # a single operator, and an 'isotropic' average of copies of it
        assert np.abs(xas[:, col] - spec_f).max() <= 1e-6 * np.abs(spec_f).max()
    p = poles[0]
    assert p["npoles"] == poles_f["npoles"]
    assert np.abs(np.array(p["alpha"][0]) - np.array(poles_f["alpha"][0])).max() < 1e-9
    assert np.abs(np.array(p["beta"][0]) - np.array(poles_f["beta"][0])).max() < 1e-9


def test_rixs_in_memory_equals_the_files(cuda, golden_dir, workdir):
    from edrixs_b200 import fedrixs, io
    src = os.path.join(golden_dir, "siam_callers")
    S, e, dm, noccu = _session(src)
    d = _drop_in(src, workdir, "rixs")
    # both paths solve the shifted systems to 1e-13 (the file path with one-RHS MINRES per
    # point, the in-memory path with the batched shifted recurrences), so that their solver
    # tolerance plays no part in the comparison
    txt = open("config.in").read().replace("linsys_tol=1e-10", "linsys_tol=1e-13").replace("linsys_max=500",
                                                                                           "linsys_max=3000")
    open("config.in", "w").write(txt)
    cfg = io.read_config("config.in")
    assert cfg["linsys_tol"] == 1e-13
    fedrixs.rixs_fsolver(0, 0, 1)
    poles_f = io.read_poles(["rixs_poles.1"])
    eloss = np.linspace(-0.5, 12.0, 500)
    spec_f = orc.spectra_from_poles(poles_f, eloss, np.full(len(eloss), 0.1), 1.0)
    Ti = _dense(os.path.join(d, "transop_rixs_i.in"), 2)
    Tf = np.conj(_dense(os.path.join(d, "transop_rixs_f.in"), 2)).T  # the file holds trans_f^+
    rixs, poles = S.rixs([cfg["omega_in"]], eloss, [(Ti, Tf)], gamma_c=cfg["gamma_in"], gamma_f=0.1, num_gs=1,
                         nkryl=cfg["nkryl"], linsys_max=cfg["linsys_max"], linsys_tol=cfg["linsys_tol"],
                         temperature=1.0)
    assert rixs.shape == (1, 500, 1)
    p = poles[0][0]
    # the pole file writes the normalisation |D_out^+ x|^2 with 10 decimals (f20.10,
    # src/io.f90:532-537); for this start vector that is ~1e-5 relative.  Compare it to the
    # file's last decimal, and the spectra with their normalisation divided out.
    nm, nf = p["norm"][0], poles_f["norm"][0]
    assert abs(nm - nf) <= 6e-11
    shape_m, shape_f = rixs[0, :, 0] / nm, spec_f / nf
    assert np.abs(shape_m - shape_f).max() <= 1e-6 * np.abs(shape_f).max()
    assert p["npoles"] == poles_f["npoles"]
    # the first coefficients, before the recurrence (no reorthogonalisation) loses orthogonality
    assert np.abs(np.array(p["alpha"][0][:10]) - np.array(poles_f["alpha"][0][:10])).max() < 1e-8
