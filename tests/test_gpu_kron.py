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
@pytest.mark.parametrize("k", [1, 2, 3, 6, 8, 13, 16, 40])
@pytest.mark.parametrize("variant", [0, 1, 2])  # automatic, staged, gather
def test_kron_spmm_equals_csr(cuda, nbath, N, mode, k, variant):
    from edrixs_b200 import device
    H, K = _both(nbath, N, mode)
    X = _rand(H.nrows, k, 7)
    want = device.spmm(H, X).cpu().numpy()
    got = K.from_slab(device.spmm(K, K.to_slab(X), col_group=variant)).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("nbath,N,mode", [(12, 6, "ham_i"), (12, 5, "ham_n"), (16, 5, "ham_i")])
@pytest.mark.parametrize("k", [1, 6, 8, 13])
def test_kron_large_slabs_gather_equals_csr(cuda, nbath, N, mode, k):
    """12 and 16 bath orbitals: slabs of up to 924 and 4,368 rows, beyond the staged ring, so
    the automatic choice is the gather product; the staged one is refused."""
    from edrixs_b200 import _lib, device
    H, K = _both(nbath, N, mode)
    assert K.max_rows > 590
    X = _rand(H.nrows, k, 11)
    want = device.spmm(H, X).cpu().numpy()
    got = K.from_slab(device.spmm(K, K.to_slab(X))).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    with pytest.raises(_lib.EdxError):
        device.spmm(K, K.to_slab(X), col_group=device.KRON_STAGED)
    V0 = _rand(H.nrows, k, 12)
    r = device.krylov(H, V0, 12)
    rk = device.krylov(K, K.to_slab(V0), 12)
    assert bool((r.neff == rk.neff).all())
    assert float((rk.alpha - r.alpha).abs().max()) <= 1e-10 * float(r.alpha.abs().max())
    assert float((rk.beta - r.beta).abs().max()) <= 1e-10 * float(r.beta.abs().max())


def test_permute_rows_round_trip(cuda):
    from edrixs_b200 import device
    H, K = _both(4, 6, "ham_i")
    X = _rand(H.nrows, 5, 2)
    assert bool((K.from_slab(K.to_slab(X)) == X).all())
    assert bool((K.to_slab(X)[:, 1] == X[K.perm, 1]).all())


@pytest.mark.parametrize("mode,k", [("ham_i", 6), ("ham_n", 6), ("ham_i", 40)])
@pytest.mark.parametrize("variant", [0, 1, 2])
def test_kron_lanczos_equals_csr(cuda, mode, k, variant):
    from edrixs_b200 import device
    H, K = _both(6, 7, mode)
    V0 = _rand(H.nrows, k, 9)
    r = device.krylov(H, V0, 30)
    rk = device.krylov(K, K.to_slab(V0), 30, apply=dict(col_group=variant))
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


@pytest.mark.parametrize("stream", [False, True])
def test_rixs_spectra_on_slab_forms_equals_csr_and_packed(cuda, stream):
    """The batched RIXS solve with H_n and H_f given only as slab forms (seeds moved into slab
    order, D_out^+ read through relabelled columns, the final-state Lanczos in the slab order
    of H_f) equals the same solve on the CSRs and on the packed forms: MINRES iterations
    identical, spectra within 1e-8 relative L-inf, the first Lanczos coefficients within
    1e-10."""
    import torch
    from edrixs_b200 import device, rixs, siam
    m, t = _model(4, 5)
    nv = m.nv
    bi, bn = device.fock_unrank(nv, 5), device.fock_unrank(nv, 6)
    Hi = device.build_csr(device.HAM_I, bi, t["hop_i"], t["coul_i"], num_val_orbs=nv)
    Hn = device.build_csr(device.HAM_N, bn, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6)
    Ki = device.kron_form(device.HAM_I, bi, t["hop_i"], t["coul_i"], num_val_orbs=nv)
    Kn = device.kron_form(device.HAM_N, bn, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6)
    assert Ki is not None and Kn is not None
    pols = siam.rixs_polarisations()
    din = [siam.text_roundtrip(siam.nonzero_terms(siam.polarised_operator(m, pols[p][0])), 2) for p in (0, 3)]
    dout = [siam.text_roundtrip(siam.nonzero_terms(np.conj(siam.polarised_operator(m, pols[p][1])).T), 2)
            for p in (0, 3)]
    Din = [device.build_csr(device.TRANS_I, bn, d, right=bi, num_val_orbs=nv, num_core_orbs=6) for d in din]
    Dout = [device.build_csr(device.TRANS_F, bi, d, right=bn, num_val_orbs=nv, num_core_orbs=6) for d in dout]
    dense = torch.sparse_csr_tensor(Hi.row_ptr, Hi.col.long(), Hi.val, (Hi.nrows, Hi.nrows)).to_dense()
    e, v = np.linalg.eigh(dense.cpu().numpy())
    gs_e, gs_v = e[:2], torch.from_numpy(np.ascontiguousarray(v[:, :2])).cuda()
    omegas = np.array([2.0, 5.0, 9.0])
    eloss = np.linspace(-0.5, 8.0, 300)
    kw = dict(nkryl=40, linsys_tol=1e-10, linsys_max=600, temperature=300.0, stream=stream, stream_window=3)
    base = dict(Hn=Hn, Hf=Hi, Din=Din, Dout=Dout, gs_e=gs_e, gs_v=gs_v)
    a = rixs.rixs_spectra(rixs.RixsProblem(**base), omegas, 0.6, eloss, 0.1, **kw)
    p = rixs.rixs_spectra(rixs.RixsProblem(**base, packed={"hn": device.pack(Hn), "hf": device.pack(Hi)}),
                          omegas, 0.6, eloss, 0.1, **kw)
    s = rixs.rixs_spectra(rixs.RixsProblem(**base, kron={"hn": Kn, "hf": Ki}), omegas, 0.6, eloss, 0.1, **kw)
    assert s.stats["hn_kron"] and s.stats["hf_kron"] and p.stats["hn_packed"] and p.stats["hf_packed"]
    assert s.stats["streamed"] == stream
    scale = np.abs(a.spectra).max()
    for r in (p, s):
        assert np.array_equal(r.iters, a.iters)
        assert np.abs(r.spectra - a.spectra).max() <= 1e-8 * scale
        assert torch.allclose(r.poles["alpha"][:, :10], a.poles["alpha"][:, :10], rtol=1e-10, atol=1e-10)
        assert torch.allclose(r.poles["norm"], a.poles["norm"], rtol=1e-12, atol=0)


def test_lowest_eigs_on_slab_form(cuda):
    """The block eigensolver with its products on the slab form (16 bath orbitals: the gather
    product) gives the CSR run's eigenvalues within 1e-9 and the same eigenvectors, returned
    in the reference's row order; the plain Lanczos edge estimate gives the lowest one too."""
    import torch
    from edrixs_b200 import solvers
    H, K = _both(16, 5, "ham_i")
    e, v = solvers.lowest_eigs(H, 3, 3, tol=1e-10)
    ek, vk = solvers.lowest_eigs(K, 3, 3, tol=1e-10)
    assert np.abs(ek - e).max() < 1e-9
    ov = torch.abs(torch.einsum("ni,ni->i", v.conj(), vk)).cpu().numpy()
    assert np.all(ov > 1 - 1e-8) or np.abs(e[1] - e[0]) < 1e-8  # degenerate pairs may rotate
    ep, _ = solvers.plain_lanczos_eigs(K, 1, 0, 400, 1e-10)
    assert abs(ep[0] - e[0]) < 1e-9


def test_understated_slab_size_is_reported_not_read_past(cuda):
    """A slab form whose max_rows understates its largest slab: the staged product clamps the
    staged boxes, the rows it holds and the hop ranks to its ring, and both the product and
    the Lanczos step report EDX_ERR_INVALID (the kernel's own range checks)."""
    import dataclasses
    from edrixs_b200 import _lib, device
    H, K = _both(10, 6, "ham_i")  # slabs of up to C(10, 5) = 252 rows
    assert K.max_rows == 252
    bad = dataclasses.replace(K, max_rows=K.max_rows // 2)
    X = _rand(H.nrows, 8, 5)
    with pytest.raises(_lib.EdxError) as e:
        device.spmm(bad, bad.to_slab(X), col_group=device.KRON_STAGED)
    assert e.value.code == 1
    with pytest.raises(_lib.EdxError) as e:
        device.krylov(bad, bad.to_slab(X), 4, apply=dict(col_group=device.KRON_STAGED))
    assert e.value.code == 1
    # the consistent form still works afterwards (the context is intact)
    want = device.spmm(H, X)
    got = K.from_slab(device.spmm(K, K.to_slab(X)))
    assert float((got - want).abs().max()) <= 1e-13 * float(want.abs().max())
