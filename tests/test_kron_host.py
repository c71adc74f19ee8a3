"""Host side of the slab (impurity x bath) form: its tables, signs and row permutation,
checked on the CPU against the oracle's CSR of the same terms (src/ham.f90:2-711).  The
numpy restatement of the slab product (kron.apply_np) must equal the CSR product for H_i
and for the core-hole H_n, on random blocks of vectors."""
import numpy as np
import pytest

from oracle import pyoracle as orc


def _terms(nbath, N, seed):
    from edrixs_b200 import siam
    m = siam.make_siam(nbath, N, seed)
    rt = siam.text_roundtrip
    return m, dict(hop_i=rt(siam.nonzero_terms(m.emat_i), 2), coul_i=rt(siam.nonzero_terms(m.umat_i), 4),
                   hop_n=rt(siam.nonzero_terms(m.emat_n), 2), coul_n=rt(siam.nonzero_terms(m.umat_n), 4))


@pytest.mark.parametrize("nbath,N,mode", [(4, 6, "ham_i"), (4, 5, "ham_n"), (6, 7, "ham_i")])
def test_slab_product_equals_csr(nbath, N, mode):
    from edrixs_b200 import kron
    m, t = _terms(nbath, N, seed=3)
    nv = m.nv
    if mode == "ham_i":
        basis = orc.fock_full_N(nv, N)
        H = orc.build_csr("ham_i", basis, t["hop_i"], t["coul_i"], num_val_orbs=nv)
        spec = kron.kron_spec(t["hop_i"], t["coul_i"], basis, "ham_i", num_val_orbs=nv)
    else:
        basis = orc.fock_full_N(nv, N + 1)
        H = orc.build_csr("ham_n", basis, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6)
        spec = kron.kron_spec(t["hop_n"], t["coul_n"], basis, "ham_n", num_val_orbs=nv, num_core_orbs=6)
    assert spec is not None and spec.nb == nbath and spec.b0 == 10
    assert spec.n == H.nrows and sorted(spec.perm) == list(range(H.nrows))
    HA = orc.build_csr("ham_i", spec.slab_full, spec.a_hop, spec.a_coul)
    assert HA.nrows == spec.nslab
    rng = np.random.default_rng(1)
    X = rng.normal(size=(H.nrows, 3)) + 1j * rng.normal(size=(H.nrows, 3))
    want = np.stack([orc.matvec(H, X[:, j]) for j in range(3)], axis=1)[spec.perm]
    got = kron.apply_np(spec, (HA.row_ptr, HA.col, HA.val), X[spec.perm])
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("nbath,N,mode", [(4, 5, "ham_n"), (6, 7, "ham_i"), (12, 3, "ham_n")])
def test_permutation_from_a_basis_tensor_equals_host(nbath, N, mode):
    """The row permutation computed with torch from a basis tensor (as the device path does,
    here on the CPU) equals the numpy one."""
    import torch
    from edrixs_b200 import kron
    m, t = _terms(nbath, N, seed=5)
    nv = m.nv
    sfx = "i" if mode == "ham_i" else "n"
    basis = orc.fock_full_N(nv, N if mode == "ham_i" else N + 1)
    kw = dict(num_val_orbs=nv, num_core_orbs=0 if mode == "ham_i" else 6)
    a = kron.kron_spec(t["hop_" + sfx], t["coul_" + sfx], basis, mode, **kw)
    b = kron.kron_spec(t["hop_" + sfx], t["coul_" + sfx], torch.from_numpy(np.asarray(basis, dtype=np.int64)), mode,
                       **kw)
    assert a is not None and b is not None and isinstance(b.perm, torch.Tensor)
    assert np.array_equal(a.perm, b.perm.numpy())


def test_no_slab_form_without_a_bath():
    """Two-body terms on every orbital (no bath): no slab form, the CSR products are used."""
    from edrixs_b200 import kron
    rng = np.random.default_rng(0)
    idx = np.array([[1, 2, 2, 1], [3, 4, 4, 3], [5, 6, 6, 5], [7, 8, 8, 7]])
    coul = (idx, rng.normal(size=4) + 0j)
    hop = (np.array([[1, 2], [2, 1]]), np.array([0.5 + 0j, 0.5 + 0j]))
    assert kron.kron_spec(hop, coul, orc.fock_full_N(8, 4), "ham_i", num_val_orbs=8) is None


def test_bath_hopping_is_refused():
    """An off-diagonal bath-bath hop has no place in the slab form (it would act inside a slab
    with a sign the tables do not carry): kron_spec declines."""
    from edrixs_b200 import kron
    m, t = _terms(4, 6, seed=3)
    idx, val = t["hop_i"]
    idx = np.vstack([idx, [[11, 12]]])
    val = np.concatenate([val, [0.3 + 0j]])
    assert kron.kron_spec((idx, val), t["coul_i"], orc.fock_full_N(m.nv, 6), "ham_i", num_val_orbs=m.nv) is None
