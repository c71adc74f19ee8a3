"""The stopping rule of the device ed_solver = 1 solver (solvers._plain_replay), replayed on
Lanczos coefficients, against the oracle's step-for-step restatement of diag_ham_lanczos
(src/lanczos.f90:6-167): same eigenvalues, same number of Krylov steps, on the 45-state known
answer (breakdown after the 11 distinct levels), on a case that converges on a check step,
and on one that never converges."""
import os

import numpy as np
import pytest

from oracle import pyoracle as orc


def _start(n, seed):
    rng = np.random.default_rng(seed)
    v1 = (rng.random(n) - 0.5).astype(np.complex128)
    return v1 / np.sqrt(np.vdot(v1, v1).real)


def _replay(csr, nev, max_niter, tol, seed, steps):
    from edrixs_b200 import solvers
    v1 = _start(csr.nrows, seed)
    a, b, _, neff = orc.build_krylov(csr, v1, steps)
    return solvers._plain_replay(a[:neff], b[:neff], neff, steps, nev, max_niter, tol)


def _known_answer(golden_dir):
    d = os.path.join(golden_dir, "known_answer")
    fock = orc.read_fock(os.path.join(d, "fock_i.in"))
    return orc.build_csr("ham_i", fock, orc.read_terms(os.path.join(d, "hopping_i.in"), 2),
                         orc.read_terms(os.path.join(d, "coulomb_i.in"), 4), num_val_orbs=20)


def test_replay_known_answer_breakdown(golden_dir):
    csr = _known_answer(golden_dir)
    e_o, _, nk_o = orc.lanczos_eigs(csr, 3, 500, 1e-8, nvec=3, seed=1)
    e, kv, nk = _replay(csr, 3, 500, 1e-8, 1, 64)
    assert nk == nk_o == 11 and kv.shape == (11, 11)
    assert np.abs(e - e_o).max() < 1e-12


def _dense_small_csr(g):
    return orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                         num_val_orbs=int(g["nv"]))


@pytest.mark.parametrize("seed", [0, 1])
def test_replay_converges_on_a_check_step(dense_small, seed):
    csr = _dense_small_csr(dense_small)
    e_o, _, nk_o = orc.lanczos_eigs(csr, 3, 500, 1e-8, nvec=2, seed=seed)
    assert _replay(csr, 3, 500, 1e-8, seed, 8) is None  # 8 steps decide nothing yet
    e, kv, nk = _replay(csr, 3, 500, 1e-8, seed, 160)
    assert nk == nk_o and nk % 10 == 0
    assert np.abs(e - e_o).max() < 1e-12


def test_replay_without_convergence(dense_small):
    csr = _dense_small_csr(dense_small)
    e_o, _, nk_o = orc.lanczos_eigs(csr, 1, 9, 1e-14, nvec=1)
    e, kv, nk = _replay(csr, 1, 9, 1e-14, 0, 9)
    assert nk == nk_o == 0 and kv is None
    assert abs(e[0] - e_o[0]) < 1e-12
