"""Block Gram-Schmidt contractions of the eigensolver (edx_gs_dot / edx_gs_update).

Bar: equal to the dense products V^H W and W - V^T C within 1e-12 relative (a different
summation order only), and deterministic (two calls give identical bits)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(1, 7, 1), (5, 1000, 3), (42, 70001, 4), (17, 5000, 8)])
def test_gs_dot_update(cuda, m, n, k):
    import torch
    from edrixs_b200 import device
    g = torch.Generator(device="cuda")
    g.manual_seed(m * 1000 + k)

    def crand(*s):
        return torch.complex(torch.randn(s, dtype=torch.float64, device="cuda", generator=g),
                             torch.randn(s, dtype=torch.float64, device="cuda", generator=g))

    Vfull = crand(m + 2, n + 5)[:, :n]   # rows with a leading dimension larger than n
    W = crand(n, k).contiguous()
    C = device.gs_dot(Vfull, m, W)
    want = Vfull[:m].conj() @ W
    assert torch.allclose(C, want, rtol=1e-12, atol=1e-12 * want.abs().max().item())
    assert torch.equal(C, device.gs_dot(Vfull, m, W))
    W2 = W.clone()
    device.gs_update(Vfull, m, W2, C)
    want2 = W - Vfull[:m].T @ C
    assert torch.allclose(W2, want2, rtol=1e-12, atol=1e-12 * want2.abs().max().item())


@pytest.mark.parametrize("n,k", [(7, 1), (70001, 3), (5000, 8)])
def test_gs_gram_rmul(cuda, n, k):
    """edx_gs_gram == W^H W and edx_gs_rmul == W M (1e-12 relative), gram deterministic."""
    import torch
    from edrixs_b200 import device
    g = torch.Generator(device="cuda")
    g.manual_seed(n + k)
    W = torch.complex(torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g),
                      torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g))
    G = device.gs_gram(W)
    want = W.conj().T @ W
    assert torch.allclose(G, want, rtol=1e-12, atol=1e-12 * want.abs().max().item())
    assert torch.equal(G, device.gs_gram(W))
    M = torch.complex(torch.randn((k, k), dtype=torch.float64, device="cuda", generator=g),
                      torch.randn((k, k), dtype=torch.float64, device="cuda", generator=g))
    want2 = W @ M
    device.gs_rmul(W, M)
    assert torch.allclose(W, want2, rtol=1e-12, atol=1e-12 * want2.abs().max().item())


def test_cholqr2_on_device(cuda):
    import torch
    from edrixs_b200 import solvers
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    W = torch.complex(torch.randn((200_000, 3), dtype=torch.float64, device="cuda", generator=g),
                      torch.randn((200_000, 3), dtype=torch.float64, device="cuda", generator=g))
    Q, R = solvers._cholqr2(W)
    R = torch.as_tensor(R).to(W.device)
    assert torch.allclose(Q.conj().T @ Q, torch.eye(3, dtype=torch.complex128, device="cuda"), atol=1e-13)
    assert torch.allclose(Q @ R, W, atol=1e-10)
