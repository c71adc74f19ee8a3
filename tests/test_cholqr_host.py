"""CholeskyQR2 of the eigensolver's tall-skinny blocks: the host logic (Cholesky factors,
the Householder fallback) on CPU tensors, with the two block passes done by torch here (on
the device they are libedx's edx_gs_gram / edx_gs_rmul, tested in test_gpu_gs.py)."""
import numpy as np
import torch


def _gram(Q):
    return Q.conj().T @ Q


def _rmul(Q, M):
    Q.copy_(Q @ torch.from_numpy(np.asarray(M)))
    return Q


def test_cholqr2_factorises_and_orthonormalises():
    from edrixs_b200.solvers import _cholqr2
    rng = np.random.default_rng(0)
    W = torch.from_numpy(rng.normal(size=(5000, 4)) + 1j * rng.normal(size=(5000, 4)))
    Q, R = _cholqr2(W, _gram, _rmul)
    assert torch.allclose(Q.conj().T @ Q, torch.eye(4, dtype=torch.complex128), atol=1e-13)
    R = torch.as_tensor(R)
    assert torch.allclose(Q @ R, W, atol=1e-11)
    assert np.allclose(np.tril(R.numpy(), -1), 0)


def test_cholqr2_falls_back_on_a_rank_deficient_block():
    from edrixs_b200.solvers import _cholqr2
    rng = np.random.default_rng(1)
    a = rng.normal(size=(3000, 1)) + 1j * rng.normal(size=(3000, 1))
    W = torch.from_numpy(np.hstack([a, 2 * a, rng.normal(size=(3000, 1))]))
    Q, R = _cholqr2(W, _gram, _rmul)   # Householder path: still a factorisation with orthonormal Q
    assert torch.allclose(Q @ R, W, atol=1e-10)
    assert torch.allclose(Q.conj().T @ Q, torch.eye(3, dtype=torch.complex128), atol=1e-12)
