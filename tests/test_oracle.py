"""Pin the CPU oracle to the reference: golden vectors made by the reference's own code.

* Fock bases == get_fock_full_N (sorted) digests at the workload sizes.
* CSR build == the reference's dense builder (manybody_operator.two_fermion/four_fermion)
  entry for entry, for H_i, H_n (core-hole sector), D_in and D_out.
* The known-answer ED case of edrixs/tests/test_fortran.py.
* Continued-fraction spectra and Boltzmann weights == get_spectra_from_poles / boltz_dist.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as orc


def test_fock_small_lists(golden_dir):
    d = json.load(open(os.path.join(golden_dir, "fock_digests.json")))
    assert list(orc.fock_full_N(4, 2)) == d["explicit_4_2"]
    assert list(orc.fock_full_N(6, 3)) == d["explicit_6_3"]


@pytest.mark.parametrize("norb,N", [(20, 10), (20, 11), (24, 12), (26, 13)])
def test_fock_digest(golden_dir, norb, N):
    d = json.load(open(os.path.join(golden_dir, "fock_digests.json")))[f"{norb}_{N}"]
    a = orc.fock_full_N(norb, N).astype("<i8")
    assert len(a) == d["ndim"]
    assert hashlib.sha256(a.tobytes()).hexdigest() == d["sha256"]


def test_binary_search_semantics():
    v = orc.fock_full_N(6, 3)
    for i, s in enumerate(v):
        assert orc.binary_search(v, s) == i + 1
    assert orc.binary_search(v, 1) == -1
    assert orc.binary_search(v, 1 << 40) == -1


def _dense_from_coo(g, name):
    shape = tuple(g[f"{name}_shape"])
    M = np.zeros(shape, dtype=complex)
    M[g[f"{name}_row"], g[f"{name}_col"]] = g[f"{name}_val"]
    return M


def _close(A, B, rtol=1e-13):
    scale = max(np.abs(B).max(), 1.0)
    return np.abs(A - B).max() <= rtol * scale


def test_build_ham_i_matches_reference_dense(dense_small):
    g = dense_small
    csr = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                        num_val_orbs=int(g["nv"]))
    ref = _dense_from_coo(g, "H_i")
    assert _close(csr.dense(), ref)
    # rows sorted ascending, no duplicate columns
    for r in range(csr.nrows):
        c = csr.col[csr.row_ptr[r]:csr.row_ptr[r + 1]]
        assert np.all(np.diff(c) > 0)


def test_build_ham_n_matches_reference_dense(dense_small):
    g = dense_small
    csr = orc.build_csr("ham_n", g["fock_n"], (g["hop_n_idx"], g["hop_n_val"]), (g["coul_n_idx"], g["coul_n_val"]),
                        num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]))
    assert csr.nrows == 6 * len(g["fock_n"])
    assert _close(csr.dense(), _dense_from_coo(g, "H_n"))


def test_build_transop_i_matches_reference_dense(dense_small):
    g = dense_small
    csr = orc.build_csr("trans_i", g["fock_n"], (g["tr_i_idx"], g["tr_i_val"]), fock_right=g["fock_i"],
                        num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]))
    assert _close(csr.dense(), _dense_from_coo(g, "D_in"))


def test_build_transop_f_matches_reference_dense(dense_small):
    g = dense_small
    csr = orc.build_csr("trans_f", g["fock_i"], (g["tr_f_idx"], g["tr_f_val"]), fock_right=g["fock_n"],
                        num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]))
    assert _close(csr.dense(), _dense_from_coo(g, "D_out"))


def test_omega_diagonal_and_sign(dense_small):
    """ham_sign = -1 with omega: A = omega*I - H exactly (rixs_driver.f90:130-133)."""
    g = dense_small
    H = orc.build_csr("ham_n", g["fock_n"], (g["hop_n_idx"], g["hop_n_val"]), (g["coul_n_idx"], g["coul_n_val"]),
                      num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]))
    z = 3.25 + 0.6j
    A = orc.build_csr("ham_n", g["fock_n"], (g["hop_n_idx"], g["hop_n_val"]), (g["coul_n_idx"], g["coul_n_val"]),
                      num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]), ham_sign=-1.0, omega=z)
    assert np.allclose(A.dense(), z * np.eye(A.nrows) - H.dense(), atol=1e-13)
    # every row carries the diagonal
    for r in range(A.nrows):
        assert r in A.col[A.row_ptr[r]:A.row_ptr[r + 1]]


def test_known_answer_eigenvalues(golden_dir):
    """edrixs/tests/test_fortran.py:8-42 through the oracle (ZHEEV path)."""
    d = os.path.join(golden_dir, "known_answer")
    fock = orc.read_fock(os.path.join(d, "fock_i.in"))
    hop = orc.read_terms(os.path.join(d, "hopping_i.in"), 2)
    coul = orc.read_terms(os.path.join(d, "coulomb_i.in"), 4)
    csr = orc.build_csr("ham_i", fock, hop, coul, num_val_orbs=20)
    e = np.linalg.eigvalsh(csr.dense())
    expected = np.loadtxt(os.path.join(d, "expected_eigvals.txt"))
    assert np.all(np.isclose(e, expected))
    assert np.abs(e - expected).max() < 1e-10


def _known_answer_hamiltonian(golden_dir):
    d = os.path.join(golden_dir, "known_answer")
    fock = orc.read_fock(os.path.join(d, "fock_i.in"))
    csr = orc.build_csr("ham_i", fock, orc.read_terms(os.path.join(d, "hopping_i.in"), 2),
                        orc.read_terms(os.path.join(d, "coulomb_i.in"), 4), num_val_orbs=20)
    return csr, np.loadtxt(os.path.join(d, "expected_eigvals.txt"))


def test_plain_lanczos_known_answer(golden_dir):
    """ed_solver = 1 (lanczos.f90:6-167) on the 45 states of test_fortran.py:8-42.

    Without reorthogonalisation a Krylov space holds one vector per distinct level, so the
    recurrence breaks down (beta < 1e-10) after as many steps as there are distinct levels
    (11), and the lowest nev eigenvalues it reports are the lowest DISTINCT levels: the
    9-fold ground level appears once. ZHEEV (ed_solver = 0) and ARPACK (ed_solver = 2) report
    it nine times."""
    csr, expected = _known_answer_hamiltonian(golden_dir)
    levels = expected[np.r_[True, np.diff(expected) > 1e-8]]
    H = csr.dense()
    e, v, nkrylov = orc.lanczos_eigs(csr, 3, 500, 1e-8, nvec=3, seed=1)
    assert nkrylov == levels.size
    assert np.abs(e - levels[:3]).max() < 1e-10
    for j in range(3):
        assert abs(np.linalg.norm(v[:, j]) - 1.0) < 1e-10
        assert np.linalg.norm(H @ v[:, j] - e[j] * v[:, j]) < 1e-10


def test_plain_lanczos_converges_on_check_steps(dense_small):
    """Convergence is tested every 10 steps on the change of the nev-th eigenvalue
    (lanczos.f90:89-110); eigenvectors come from re-running the recurrence (:133-157)."""
    g = dense_small
    csr = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                        num_val_orbs=int(g["nv"]))
    H = csr.dense()
    exact = np.linalg.eigvalsh(H)
    for seed in (0, 1):
        e, v, nkrylov = orc.lanczos_eigs(csr, 3, 500, 1e-8, nvec=2, seed=seed)
        assert nkrylov % 10 == 0 and nkrylov < csr.nrows
        assert np.abs(e - exact[:3]).max() < 1e-9
        for j in range(2):
            assert np.linalg.norm(H @ v[:, j] - e[j] * v[:, j]) < 1e-8
        # the start vector is real: so are the Lanczos vectors of this real symmetric H
        if np.abs(H.imag).max() == 0:
            assert np.abs(v.imag).max() == 0


def test_plain_lanczos_without_convergence_gives_zero_vectors(dense_small):
    """When max_niter passes before the test succeeds, nkrylov stays 0 in the reference and the
    eigenvector pass (lanczos.f90:133-157) runs no step: the vectors are zero, the eigenvalues
    those of the last check."""
    g = dense_small
    csr = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                        num_val_orbs=int(g["nv"]))
    e, v, nkrylov = orc.lanczos_eigs(csr, 1, 9, 1e-14, nvec=1)
    assert nkrylov == 0 and not v.any()
    assert e[0] > np.linalg.eigvalsh(csr.dense())[0]


def test_spectra_and_boltzmann(golden_dir):
    with np.load(os.path.join(golden_dir, "spectra.npz")) as z:
        g = {k: z[k] for k in z.files}
    poles = {"npoles": list(g["npoles"]), "eigval": list(g["eigval"]), "norm": list(g["norm"]),
             "alpha": [list(a) for a in g["alpha"]], "beta": [list(b) for b in g["beta"]]}
    s = orc.spectra_from_poles(poles, g["om_xas"], 0.3, 300.0)
    assert np.abs(s - g["s_xas"]).max() <= 1e-12 * np.abs(g["s_xas"]).max()
    s = orc.spectra_from_poles(poles, g["om_rixs"], g["gam_rixs"], 10.0)
    assert np.abs(s - g["s_rixs"]).max() <= 1e-12 * np.abs(g["s_rixs"]).max()
    for T, w in zip(g["boltz_T"], g["boltz"]):
        assert np.allclose(orc.boltz_dist(g["boltz_e"], T), w, rtol=1e-14, atol=0)


def test_matvec_krylov_minres_consistency(dense_small):
    """Oracle SpMV / Krylov / MINRES against dense numpy algebra on the same matrix."""
    g = dense_small
    H = orc.build_csr("ham_n", g["fock_n"], (g["hop_n_idx"], g["hop_n_val"]), (g["coul_n_idx"], g["coul_n_val"]),
                      num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]))
    Hd = H.dense()
    rng = np.random.default_rng(0)
    x = rng.normal(size=H.nrows) + 1j * rng.normal(size=H.nrows)
    assert np.allclose(orc.matvec(H, x), Hd @ x, rtol=1e-13, atol=1e-12)
    a, b, nrm, neff = orc.build_krylov(H, x, 20)
    assert neff == 20 and abs(nrm - np.vdot(x, x).real) < 1e-9
    # first alpha is the Rayleigh quotient of the start vector
    assert abs(a[0] - np.vdot(x, Hd @ x).real / np.vdot(x, x).real) < 1e-9
    z = 40.0 + 0.6j
    A = orc.build_csr("ham_n", g["fock_n"], (g["hop_n_idx"], g["hop_n_val"]), (g["coul_n_idx"], g["coul_n_val"]),
                      num_val_orbs=int(g["nv"]), num_core_orbs=int(g["nc"]), ham_sign=-1.0, omega=z)
    sol, it, res = orc.minres(A, x, 1e-10, 2000)
    exact = np.linalg.solve(A.dense(), x)
    assert np.abs(sol - exact).max() / np.abs(exact).max() < 1e-8
    assert res <= 1e-10


def test_denmat_oracle_trace(dense_small):
    g = dense_small
    H = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                      num_val_orbs=int(g["nv"]))
    e, v = np.linalg.eigh(H.dense())
    dm = orc.denmat(g["fock_i"], int(g["nv"]), v[:, 0])
    assert abs(np.trace(dm).real - int(g["nelec"])) < 1e-10
    assert np.allclose(dm, dm.conj().T, atol=1e-10)


def test_denmat_matches_reference_two_fermion(dense_small, golden_dir):
    """<c+_i c_j> of the two lowest eigenstates of the dense_small H_i: the oracle's restatement
    of ed_driver.f90:194-248 against every operator built by the reference's
    manybody_operator.two_fermion (tests/golden/denmat.npz).  Eigenvector phases cancel; the
    reference skips rows with |v_a| < 1e-10 in the off-diagonals, so 1e-9 absolute."""
    g = dense_small
    nv = int(g["nv"])
    csr = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                        num_val_orbs=nv)
    e, v = np.linalg.eigh(csr.dense())
    with np.load(os.path.join(golden_dir, "denmat.npz")) as z:
        rho, ev = z["rho"], z["eigvals"]
    assert np.allclose(e[:3], ev, atol=1e-12)
    for k in range(2):
        got = orc.denmat(g["fock_i"], nv, v[:, k])
        assert np.allclose(got, rho[k], atol=1e-9, rtol=0)
        assert abs(np.trace(got).real - int(g["nelec"])) < 1e-9


def _opavg_case(dense_small, golden_dir, d):
    """A working directory for opavg: the d-electron number operator (orbitals 1..10) as
    hopping_i.in, no Coulomb terms, the dense_small basis and its two lowest eigenvectors.
    Returns the expected <N_d> from the reference two_fermion density matrices."""
    from edrixs_b200 import io as edxio
    g = dense_small
    nv = int(g["nv"])
    csr = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                        num_val_orbs=nv)
    e, v = np.linalg.eigh(csr.dense())
    E = np.zeros((nv, nv), dtype=complex)
    E[:10, :10] = np.eye(10)
    edxio.write_emat(E, os.path.join(d, "hopping_i.in"))
    edxio.write_umat(np.zeros((nv,) * 4, dtype=complex), os.path.join(d, "coulomb_i.in"))
    edxio.write_fock(os.path.join(d, "fock_i.in"), g["fock_i"])
    edxio.write_config(d, num_val_orbs=nv, num_core_orbs=0, num_gs=2)
    for k in range(2):
        edxio.write_eigvec(os.path.join(d, f"eigvec.{k + 1}"), e[k], v[:, k])
    with np.load(os.path.join(golden_dir, "denmat.npz")) as z:
        rho = z["rho"]
    return e[:2], np.array([np.trace(rho[k][:10, :10]) for k in range(2)])


def test_opavg_matches_reference_two_fermion(dense_small, golden_dir, tmp_path):
    """opavg_driver.f90 restated: <v|N_d|v> of two eigenvectors equals the trace over the d
    orbitals of the reference's two_fermion density matrices."""
    from oracle import drivers as odrv
    e, want = _opavg_case(dense_small, golden_dir, str(tmp_path))
    ev, got = odrv.opavg(str(tmp_path))
    assert np.allclose(ev, e, atol=1e-14)
    assert np.allclose(got, want, atol=1e-12)
    assert np.all(np.abs(got.imag) < 1e-13)


def test_opavg_file_format(tmp_path):
    """write_opavg = src/io.f90:638-659: i5, then eigenvalue, Re and Im as f20.10."""
    from edrixs_b200 import io as edxio
    p = str(tmp_path / "opavg.dat")
    edxio.write_opavg(p, [-12.5, 3.0], [complex(2.25, -0.0), -1.0 + 1e-12j])  # negative zero keeps its sign
    lines = open(p).read().splitlines()
    assert lines[0] == "    1" + "{:20.10f}".format(-12.5) + "{:20.10f}".format(2.25) + "{:20.10f}".format(-0.0)
    assert len(lines[1]) == 65 and lines[1].startswith("    2")


def test_oracle_ed_driver_follows_ed_solver_1(golden_dir, tmp_path):
    """drivers.ed(follow_ed_solver=True) on the known-answer files with ed_solver = 1 and
    min_ndim below the dimension: the plain Lanczos path of ed_driver.f90:154-158."""
    import shutil
    from oracle import drivers as odrv
    d = tmp_path / "ka"
    shutil.copytree(os.path.join(golden_dir, "known_answer"), d)
    (d / "config.in").write_text("&control\ned_solver=1\nnum_val_orbs=20\nneval=3\nnvector=2\n"
                                 "maxiter=500\neigval_tol=1e-10\nmin_ndim=10\n&end\n")
    expected = np.loadtxt(d / "expected_eigvals.txt")
    levels = expected[np.r_[True, np.diff(expected) > 1e-8]]
    e, v, H, fock, cfg = odrv.ed(str(d), follow_ed_solver=True)
    assert np.abs(e - levels[:3]).max() < 1e-10 and v.shape == (45, 2)
    e0, _, _, _, _ = odrv.ed(str(d))
    assert np.abs(e0 - expected[:3]).max() < 1e-10    # dense: the 9-fold level three times
