"""Parity with the oracle at the benchmark workloads' own sizes.

The other GPU parity tests use models of at most 16 valence orbitals.  These run the same
comparisons on the matrices the benchmark and the configurations use:

* the 20-orbital, N = 10 ground sector: H_i with 184,756 rows (11.2 M nonzeros);
* the N_v = 11 one-core-hole intermediate sector: H_n with 1,007,760 rows (68.3 M
  nonzeros), built with ham_sign = +1 and with ham_sign = -1 and a complex omega (the
  reference's MINRES matrix, src/rixs_driver.f90:130-133);
* the transition operators D_in (1,007,760 x 184,756) and D_out (184,756 x 1,007,760) of
  both incoming and both outgoing polarisations.

Bar: CSR row pointers, columns and value bits identical to the oracle (src/ham.f90:2-1115,
src/m_types.f90:74-121); the lowest 4 eigenvalues of H_i within 1e-10 eV of the oracle's
ARPACK-family solver (src/arpack.f90:2-112); the first 20 Lanczos coefficients of the XAS
recurrence on H_n (src/lanczos.f90:210-303) within 1e-8 relative.
"""
import numpy as np
import pytest

from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu

NV, N, NCORE = 20, 10, 6


@pytest.fixture(scope="module")
def work():
    import bench
    from edrixs_b200 import siam
    m, t = bench.workload_terms(NV - 10, N)
    t["xas"] = [siam.text_roundtrip(siam.nonzero_terms(siam.polarised_operator(m, p)), 2)
                for p in siam.atomic()["xas_polvec"][:2]]
    return m, t, orc.fock_full_N(NV, N), orc.fock_full_N(NV, N + 1)


def _assert_bitexact(gpu, ref):
    assert gpu.nrows == ref.nrows and gpu.nnz == ref.nnz
    assert np.array_equal(gpu.row_ptr.cpu().numpy(), ref.row_ptr)
    assert np.array_equal(gpu.col.cpu().numpy(), ref.col)
    assert np.array_equal(gpu.val.cpu().numpy().view(np.float64), ref.val.view(np.float64))


def test_c0_H_i_184756_rows_bitexact(cuda, work):
    from edrixs_b200 import device
    m, t, fi, fn = work
    ref = orc.build_csr("ham_i", fi, t["hop_i"], t["coul_i"], num_val_orbs=NV)
    assert ref.nrows == 184756
    H = device.build_csr(device.HAM_I, device.fock_unrank(NV, N), t["hop_i"], t["coul_i"], num_val_orbs=NV)
    _assert_bitexact(H, ref)


@pytest.mark.parametrize("ham_sign,omega", [(1.0, 0j), (-1.0, 7.25 + 0.6j)], ids=["sign+1", "sign-1_omega"])
def test_c2_H_n_1007760_rows_bitexact(cuda, work, ham_sign, omega):
    from edrixs_b200 import device
    m, t, fi, fn = work
    ref = orc.build_csr("ham_n", fn, t["hop_n"], t["coul_n"], num_val_orbs=NV, num_core_orbs=NCORE,
                        ham_sign=ham_sign, omega=omega)
    assert ref.nrows == 1007760
    H = device.build_csr(device.HAM_N, device.fock_unrank(NV, N + 1), t["hop_n"], t["coul_n"], num_val_orbs=NV,
                         num_core_orbs=NCORE, ham_sign=ham_sign, omega=omega)
    _assert_bitexact(H, ref)


def test_c2_D_in_D_out_1007760x184756_bitexact(cuda, work):
    from edrixs_b200 import device
    m, t, fi, fn = work
    bi, bn = device.fock_unrank(NV, N), device.fock_unrank(NV, N + 1)
    for d in t["din"]:
        ref = orc.build_csr("trans_i", fn, d, fock_right=fi, num_val_orbs=NV, num_core_orbs=NCORE)
        assert (ref.nrows, ref.ncols) == (1007760, 184756)
        _assert_bitexact(device.build_csr(device.TRANS_I, bn, d, right=bi, num_val_orbs=NV, num_core_orbs=NCORE),
                         ref)
    for d in t["dout"]:
        ref = orc.build_csr("trans_f", fi, d, fock_right=fn, num_val_orbs=NV, num_core_orbs=NCORE)
        assert (ref.nrows, ref.ncols) == (184756, 1007760)
        _assert_bitexact(device.build_csr(device.TRANS_F, bi, d, right=bn, num_val_orbs=NV, num_core_orbs=NCORE),
                         ref)


@pytest.fixture(scope="module")
def c0_ground(work):
    m, t, fi, fn = work
    Hf = orc.build_csr("ham_i", fi, t["hop_i"], t["coul_i"], num_val_orbs=NV)
    e, v = orc.ed_eigs(Hf, 4, dense_below=0, tol=1e-13)
    return Hf, e, v


def test_c0_lowest4_eigenvalues_184756_rows_1e10(cuda, work, c0_ground):
    from edrixs_b200 import device, solvers
    m, t, fi, fn = work
    Hf, e_ref, _ = c0_ground
    H = device.build_csr(device.HAM_I, device.fock_unrank(NV, N), t["hop_i"], t["coul_i"], num_val_orbs=NV)
    e, v = solvers.lowest_eigs(H, 4, 4, tol=1e-10, packed=device.pack(H))
    e = np.asarray(e)
    assert np.abs(e - e_ref).max() <= 1e-10, (e, e_ref)
    # and the vectors are eigenvectors of the oracle's matrix
    vh = v.cpu().numpy()
    for j in range(4):
        r = orc.matvec(Hf, vh[:, j]) - e[j] * vh[:, j]
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(vh[:, j])


def test_c0_xas_krylov_first20_on_H_n_1007760_rows_1e8(cuda, work, c0_ground):
    import torch
    from edrixs_b200 import device
    m, t, fi, fn = work
    _, _, v = c0_ground
    Hn_ref = orc.build_csr("ham_n", fn, t["hop_n"], t["coul_n"], num_val_orbs=NV, num_core_orbs=NCORE)
    Hn = device.build_csr(device.HAM_N, device.fock_unrank(NV, N + 1), t["hop_n"], t["coul_n"], num_val_orbs=NV,
                          num_core_orbs=NCORE)
    Pn = device.pack(Hn)
    for pol, d in enumerate(t["xas"]):
        D = orc.build_csr("trans_i", fn, d, fock_right=fi, num_val_orbs=NV, num_core_orbs=NCORE)
        phi = orc.matvec(D, v[:, 0])
        a_ref, b_ref, nrm_ref, neff_ref = orc.build_krylov(Hn_ref, phi, 20)
        assert neff_ref == 20
        for A in (Hn, Pn):  # the CSR product and the packed product the batched path runs
            r = device.krylov(A, torch.from_numpy(phi).cuda().reshape(-1, 1), 20)
            assert int(r.neff[0]) == 20
            a = r.alpha[0, :20].cpu().numpy()
            b = r.beta[0, :20].cpu().numpy()
            assert np.abs(a - a_ref).max() <= 1e-8 * np.abs(a_ref).max(), (pol, a, a_ref)
            assert np.abs(b - b_ref).max() <= 1e-8 * np.abs(b_ref).max(), (pol, b, b_ref)
            assert abs(float(r.norm[0]) - nrm_ref) <= 1e-12 * nrm_ref
