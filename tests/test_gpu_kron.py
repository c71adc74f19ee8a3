"""The slab (impurity x bath) product against the CSR product of the same Hamiltonian.

edx_kron_spmm (Y = H X in slab order) and edx_krylov with apply_kron (the fused Lanczos step
of src/lanczos.f90:210-303 on the slab form) must give the CSR product's results
(src/spmv.f90:73-103 on the bit-exact build of src/ham.f90:2-711) up to the summation order:
products within 1e-13 relative, Lanczos coefficients within 1e-10.  Small impurity models
for every column-group width, then the benchmark's own H_i (184,756 rows) and core-hole H_n
(1,007,760 rows).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(nbath, N, seed=3):
    from edrixs_b200 import siam
    m = siam.make_siam(nbath, N, seed)
    rt = siam.text_roundtrip
    return m, dict(hop_i=rt(siam.nonzero_terms(m.emat_i), 2), coul_i=rt(siam.nonzero_terms(m.umat_i), 4),
                   hop_n=rt(siam.nonzero_terms(m.emat_n), 2), coul_n=rt(siam.nonzero_terms(m.umat_n), 4))


def _both(nbath, N, mode):
    from edrixs_b200 import device
    m, t = _model(nbath, N)
    nv = m.nv
    if mode == "ham_i":
        b = device.fock_unrank(nv, N)
        H = device.build_csr(device.HAM_I, b, t["hop_i"], t["coul_i"], num_val_orbs=nv)
        K = device.kron_form(device.HAM_I, b, t["hop_i"], t["coul_i"], num_val_orbs=nv)
    else:
        b = device.fock_unrank(nv, N + 1)
        H = device.build_csr(device.HAM_N, b, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6)
        K = device.kron_form(device.HAM_N, b, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6)
    assert K is not None and K.nrows == H.nrows
    return H, K


def _rand(n, k, seed):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    re = torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g)
    im = torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g)
    return torch.complex(re, im).contiguous()


@pytest.mark.parametrize("nbath,N,mode", [(4, 6, "ham_i"), (4, 5, "ham_n"), (6, 7, "ham_i"), (6, 7, "ham_n")])
@pytest.mark.parametrize("k,cw", [(1, 0), (2, 0), (3, 0), (6, 0), (8, 0), (13, 0), (16, 0), (40, 0)])
def test_kron_spmm_equals_csr(cuda, nbath, N, mode, k, cw):
    from edrixs_b200 import device
    H, K = _both(nbath, N, mode)
    X = _rand(H.nrows, k, 7)
    want = device.spmm(H, X).cpu().numpy()
    got = K.from_slab(device.spmm(K, K.to_slab(X), col_group=cw)).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_permute_rows_round_trip(cuda):
    from edrixs_b200 import device
    H, K = _both(4, 6, "ham_i")
    X = _rand(H.nrows, 5, 2)
    assert bool((K.from_slab(K.to_slab(X)) == X).all())
    assert bool((K.to_slab(X)[:, 1] == X[K.perm, 1]).all())


@pytest.mark.parametrize("mode,k", [("ham_i", 6), ("ham_n", 6), ("ham_i", 40)])
def test_kron_lanczos_equals_csr(cuda, mode, k):
    from edrixs_b200 import device
    H, K = _both(6, 7, mode)
    V0 = _rand(H.nrows, k, 9)
    r = device.krylov(H, V0, 30)
    rk = device.krylov(K, K.to_slab(V0), 30)
    assert bool((r.neff == rk.neff).all())
    a, ak = r.alpha.cpu().numpy(), rk.alpha.cpu().numpy()
    b, bk = r.beta.cpu().numpy(), rk.beta.cpu().numpy()
    assert np.abs(ak - a).max() <= 1e-10 * np.abs(a).max()
    assert np.abs(bk - b).max() <= 1e-10 * np.abs(b).max()
    assert np.allclose(rk.norm.cpu().numpy(), r.norm.cpu().numpy(), rtol=1e-13)


def test_kron_workload_sizes(cuda):
    """The benchmark's matrices: H_i (184,756 rows) at 768 columns and H_n (1,007,760 rows) at
    6 columns, products and 8 Lanczos steps, against the CSR products."""
    import bench
    from edrixs_b200 import device
    m, t = bench.workload_terms(10, 10)
    nv = m.nv
    bi, bn = device.fock_unrank(nv, 10), device.fock_unrank(nv, 11)
    cases = [(device.HAM_I, bi, t["hop_i"], t["coul_i"], 0, 768, 184756),
             (device.HAM_N, bn, t["hop_n"], t["coul_n"], 6, 6, 1007760)]
    for mode, b, hop, coul, nc, k, n in cases:
        H = device.build_csr(mode, b, hop, coul, num_val_orbs=nv, num_core_orbs=nc)
        K = device.kron_form(mode, b, hop, coul, num_val_orbs=nv, num_core_orbs=nc)
        assert K is not None and K.nrows == n == H.nrows
        X = _rand(n, k, 4)
        want = device.spmm(H, X)
        got = K.from_slab(device.spmm(K, K.to_slab(X)))
        scale = float(want.abs().max())
        assert float((got - want).abs().max()) <= 1e-13 * scale
        del want, got
        r = device.krylov(H, X, 8)
        rk = device.krylov(K, K.to_slab(X), 8)
        assert bool((r.neff == rk.neff).all())
        assert float((rk.alpha - r.alpha).abs().max()) <= 1e-10 * float(r.alpha.abs().max())
        assert float((rk.beta - r.beta).abs().max()) <= 1e-10 * float(r.beta.abs().max())
