"""The drop-in solvers' host logic on the CPU: file reading and writing, the order of the
phases, the ground-state loop and the pole files, with a stand-in for the device layer.

The stand-in (below) answers every edrixs_b200.device call the drop-in makes with the
oracle's CPU arithmetic, so these tests need no GPU.  They do not test the CUDA path (the
-m gpu tests do, on the same files); they test what sits around it.  The inputs are the
files the reference's 1v1c callers wrote for a d8 ion (tests/golden/kh_1v1c), and the
spectra must equal the reference's Kramers-Heisenberg answers as the oracle drivers' do."""
import os
import shutil
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from edrixs_b200 import device, fedrixs, solvers, trace
from edrixs_b200 import io as edxio
from oracle import pyoracle as orc

KH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kh_1v1c")
MODES = {device.HAM_I: "ham_i", device.HAM_N: "ham_n", device.TRANS_I: "trans_i", device.TRANS_F: "trans_f"}


@pytest.fixture
def host_device(monkeypatch):
    """edrixs_b200.device and the eigensolvers answered on the CPU by the oracle."""
    def build_csr(mode, left, hopping, coulomb=None, right=None, num_val_orbs=0, num_core_orbs=0, **kw):
        return orc.build_csr(MODES[mode], left.states, hopping, coulomb,
                             fock_right=None if right is None else right.states, num_val_orbs=num_val_orbs,
                             num_core_orbs=num_core_orbs)

    def spmm(A, X):
        X = X.reshape(X.shape[0], -1).numpy()
        return torch.from_numpy(np.stack([orc.matvec(A, X[:, j]) for j in range(X.shape[1])], axis=1))

    def krylov(A, V0, maxn):
        V0 = V0.reshape(V0.shape[0], -1).numpy()
        k = V0.shape[1]
        al, be = np.zeros((k, maxn)), np.zeros((k, maxn))
        nrm, neff = np.zeros(k), np.zeros(k, dtype=np.int32)
        for j in range(k):
            a, b, nrm[j], neff[j] = orc.build_krylov(A, V0[:, j], maxn)
            al[j, :neff[j]], be[j, :neff[j]] = a, b
        return SimpleNamespace(alpha=torch.from_numpy(al), beta=torch.from_numpy(be), norm=torch.from_numpy(nrm),
                               neff=torch.from_numpy(neff))

    def minres(A, b, tol, maxit, alpha=1.0, sigma=0.0):
        M = alpha * A.dense() + sigma * np.eye(A.nrows)
        return torch.from_numpy(np.linalg.solve(M, b.numpy())), 1, 0.0

    def denmat(basis, nv, v):
        v = v.reshape(v.shape[0], -1).numpy()
        return torch.from_numpy(np.stack([orc.denmat(basis.states, nv, v[:, k]) for k in range(v.shape[1])]))

    def eigs(H, nev, nvec=None, **kw):
        e, v = np.linalg.eigh(H.dense())
        return e[:nev], torch.from_numpy(v[:, :max(nev, nvec or nev)])

    monkeypatch.setattr(device, "require_cuda", lambda: None)
    monkeypatch.setattr(device, "basis_from_states",
                        lambda s: SimpleNamespace(states=np.asarray(s).astype(np.int64), ndim=len(s)))
    monkeypatch.setattr(device, "build_csr", build_csr)
    monkeypatch.setattr(device, "spmm", spmm)
    monkeypatch.setattr(device, "krylov", krylov)
    monkeypatch.setattr(device, "minres", minres)
    monkeypatch.setattr(device, "denmat", denmat)
    monkeypatch.setattr(device, "pack", lambda H: None)
    monkeypatch.setattr(solvers, "dense_eigs", lambda H, nev: eigs(H, nev))
    monkeypatch.setattr(solvers, "lowest_eigs", eigs)
    monkeypatch.setattr(torch.Tensor, "cuda", lambda self, *a, **k: self)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    level = trace._level
    trace.enable(1)
    trace.records.clear()
    yield
    trace.enable(level)
    trace.records.clear()


def _workdir(tmp_path, name):
    d = tmp_path / name
    d.mkdir()
    for src in (os.path.join(KH, "ed_00"), os.path.join(KH, name)):
        for fn in os.listdir(src):
            shutil.copy(os.path.join(src, fn), d / fn)
    return d


def test_drop_in_host_logic_reproduces_kramers_heisenberg(host_device, tmp_path, monkeypatch):
    with np.load(os.path.join(KH, "kh_spectra.npz")) as z:
        g = {k: z[k] for k in z.files}
    T = float(g["temperature"])
    # ED: eigvals.dat, denmat.dat; then eigvec.1 for the next steps
    d = _workdir(tmp_path, "ed_00")
    monkeypatch.chdir(d)
    fedrixs.ed_fsolver(fedrixs.FakeComm().py2f(), 0, 1)
    ev = np.loadtxt(d / "eigvals.dat", ndmin=2)
    assert ev.shape == (3, 2) and np.allclose(ev[:, 1], g["eval_i"][:3], atol=1e-9)
    dm = np.loadtxt(d / "denmat.dat", ndmin=2)
    assert dm.shape == (100, 5) and abs(dm[::11, 3].sum() - 8.0) < 1e-8    # trace = 8 electrons (d8)
    H = orc.build_csr("ham_i", orc.read_fock(str(d / "fock_i.in")), orc.read_terms(str(d / "hopping_i.in"), 2),
                      orc.read_terms(str(d / "coulomb_i.in"), 4), num_val_orbs=10)
    e, v = np.linalg.eigh(H.dense())

    def with_gs(name):
        w = _workdir(tmp_path, name)
        edxio.write_eigvec(str(w / "eigvec.1"), e[0], v[:, 0])
        monkeypatch.chdir(w)
        return w

    for ip, name in enumerate(["xas_01", "xas_02"]):
        w = with_gs(name)
        fedrixs.xas_fsolver(0, 0, 1)
        spec = orc.spectra_from_poles(edxio.read_poles([str(w / "xas_poles.1")]), g["ominc"],
                                      float(g["gamma_c_xas"]), T)
        ref = g["xas"][:, ip]
        # the pole file carries alpha and beta to 10 decimals (src/io.f90:532-537)
        assert np.abs(spec - ref).max() <= 1e-7 * np.abs(ref).max()
    npol = g["rixs"].shape[2]
    for k, name in enumerate(["rixs_03", "rixs_04"]):
        w = with_gs(name)
        fedrixs.rixs_fsolver(0, 0, 1)
        spec = orc.spectra_from_poles(edxio.read_poles([str(w / "rixs_poles.1")]), g["eloss"], float(g["gamma_f"]), T)
        ref = g["rixs"][k // npol, :, k % npol]
        assert np.abs(spec - ref).max() <= 1e-7 * np.abs(ref).max()
    # opavg: <v|H|v> of the ground state is its energy
    w = tmp_path / "opavg"
    shutil.copytree(os.path.join(KH, "ed_00"), w)
    edxio.write_eigvec(str(w / "eigvec.1"), e[0], v[:, 0])
    monkeypatch.chdir(w)
    fedrixs.opavg_fsolver(0, 0, 1)
    avg = np.loadtxt(w / "opavg.dat", ndmin=2)
    assert abs(avg[0, -2] - e[0]) < 1e-9
    # every phase of every solver was traced, in order
    names = [r["phase"] for r in trace.records]
    assert names[:3] == ["ed: build H_i", "ed: eigenpairs", "ed: density matrix"]
    assert names.count("xas: Krylov") == 2 and names.count("rixs: MINRES") == 2
    assert names[-1] == "opavg: build O, <v|O|v>" and all(r["ok"] for r in trace.records)


def test_drop_in_host_logic_on_two_valence_shell_files(host_device, tmp_path, monkeypatch):
    """The same on the files of the reference's 2v1c callers (t2g + p shells, an s core of two
    orbitals, a quadrupolar operator; tests/golden/callers_2v1c), against the exact spectra of
    the matrices the reference's two_fermion / four_fermion build from them."""
    G = os.path.join(os.path.dirname(KH), "callers_2v1c")
    with np.load(os.path.join(G, "dense.npz")) as z:
        d = {k: z[k] for k in z.files}
    M = {}
    for key in d:
        if key.endswith("_shape"):
            name = key[:-6]
            M[name] = np.zeros(tuple(d[key]), dtype=complex)
            M[name][d[name + "_row"], d[name + "_col"]] = d[name + "_val"]

    def exact(H, phi, e0, om, gam):
        ev, U = np.linalg.eigh(H)
        w2 = np.abs(U.conj().T @ phi) ** 2
        return -np.imag((w2[None, :] / (om[:, None] + 1j * gam + e0 - ev[None, :])).sum(axis=1)) / np.pi

    def workdir(name, e0=None, g0=None):
        w = tmp_path / name
        w.mkdir()
        for src in {os.path.join(G, "ed_00"), os.path.join(G, name)}:
            if os.path.isdir(src):
                for fn in os.listdir(src):
                    shutil.copy(os.path.join(src, fn), w / fn)
        if g0 is not None:
            edxio.write_eigvec(str(w / "eigvec.1"), e0, g0)
        monkeypatch.chdir(w)
        return w

    w = workdir("ed_00")
    fedrixs.ed_fsolver(0, 0, 1)
    e, v = np.linalg.eigh(M["H_i"])
    assert np.allclose(np.loadtxt(w / "eigvals.dat", ndmin=2)[:, 1], e[:2], atol=1e-9)
    om = np.linalg.eigvalsh(M["H_n"])[0] - e[0] + np.linspace(-3.0, 12.0, 151)
    for name in ("xas_01", "xas_02"):
        w = workdir(name, e[0], v[:, 0])
        fedrixs.xas_fsolver(0, 0, 1)
        spec = orc.spectra_from_poles(edxio.read_poles([str(w / "xas_poles.1")]), om, 0.3, 1.0)
        ref = exact(M["H_n"], M[f"D_{name}"] @ v[:, 0], e[0], om, 0.3)
        assert np.abs(spec - ref).max() <= 1e-7 * np.abs(ref).max()
    eloss = np.linspace(-0.5, 6.0, 66)
    for name in ("rixs_03", "rixs_04"):
        w = workdir(name, e[0], v[:, 0])
        cfg = edxio.read_config(str(w / "config.in"))
        fedrixs.rixs_fsolver(0, 0, 1)
        poles = edxio.read_poles([str(w / "rixs_poles.1")])
        spec = orc.spectra_from_poles(poles, eloss, 0.1, 1.0)
        z = cfg["omega_in"] + e[0] + 1j * cfg["gamma_in"]
        x = np.linalg.solve(z * np.eye(len(M["H_n"])) - M["H_n"], M[f"D_in_{name}"] @ v[:, 0])
        ref = exact(M["H_i"], M[f"D_out_{name}"] @ x, e[0], eloss, 0.1)
        # off resonance the norm is small, and the file carries it to 10 decimals
        # (src/io.f90:532-537): a relative error of up to 5e-11 / norm comes from the format
        tol = 1e-7 + 5e-11 / poles["norm"][0]
        assert np.abs(spec - ref).max() <= tol * np.abs(ref).max()


def test_command_line_entry_points(host_device, tmp_path, monkeypatch, capsys):
    """`python -m edrixs_b200.scripts ed|xas|rixs|opavg` (the ed.x ... opavg.x of the reference,
    setup.py:101-108) run the drop-in solvers in the working directory; a nonzero RANK runs
    nothing; a bad command prints the usage and returns 2."""
    from edrixs_b200 import scripts
    d = _workdir(tmp_path, "ed_00")
    monkeypatch.chdir(d)
    monkeypatch.setenv("RANK", "1")
    assert scripts.main(["ed"]) == 0 and not (d / "eigvals.dat").exists()
    monkeypatch.setenv("RANK", "0")
    assert scripts.main(["ed"]) == 0 and (d / "eigvals.dat").exists() and (d / "denmat.dat").exists()
    assert scripts.main(["bogus"]) == 2 and "usage" in capsys.readouterr().err
