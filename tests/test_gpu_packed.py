"""Packed form (edx_pack_*) and the Lanczos product on it.

Bar: packing is lossless, so unpacking gives back the CSR's off-diagonal columns in CSR
order and bit-identical values, plus the diagonal.  The Lanczos coefficients on the packed
product match the oracle to the CSR product's tolerance (rtol 1e-8) and the CSR product to
1e-10 relative.
"""
import numpy as np
import pytest

from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu


def _ham(mode="ham_i", nbath=6, N=8, seed=5):
    from edrixs_b200 import device, siam
    m = siam.make_siam(nbath, N, seed)
    nv = m.nv
    if mode == "ham_i":
        hop = siam.text_roundtrip(siam.nonzero_terms(m.emat_i), 2)
        coul = siam.text_roundtrip(siam.nonzero_terms(m.umat_i), 4)
        ref = orc.build_csr("ham_i", orc.fock_full_N(nv, N), hop, coul, num_val_orbs=nv)
        gpu = device.build_csr(device.HAM_I, device.fock_unrank(nv, N), hop, coul, num_val_orbs=nv)
    else:
        hop = siam.text_roundtrip(siam.nonzero_terms(m.emat_n), 2)
        coul = siam.text_roundtrip(siam.nonzero_terms(m.umat_n), 4)
        ref = orc.build_csr("ham_n", orc.fock_full_N(nv, N + 1), hop, coul, num_val_orbs=nv, num_core_orbs=6)
        gpu = device.build_csr(device.HAM_N, device.fock_unrank(nv, N + 1), hop, coul, num_val_orbs=nv,
                               num_core_orbs=6)
    return ref, gpu


def _assert_pack_lossless(P, A):
    rp, col, val = A.row_ptr.cpu().numpy(), A.col.cpu().numpy(), A.val.cpu().numpy()
    prp, pcol, pval = (t.cpu().numpy() for t in P.unpack())
    diag = P.diag.cpu().numpy()
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    off = col != rows
    assert np.array_equal(prp, np.r_[0, np.cumsum(np.bincount(rows[off], minlength=len(rp) - 1))])
    assert np.array_equal(pcol, col[off])
    assert np.array_equal(pval.view(np.float64), val[off].view(np.float64))
    d = np.zeros(len(rp) - 1, dtype=np.complex128)
    d[rows[~off]] = val[~off]
    assert np.array_equal(diag.view(np.float64), d.view(np.float64))


@pytest.mark.parametrize("form", ["auto", "wide"])
@pytest.mark.parametrize("mode", ["ham_i", "ham_n"])
def test_pack_is_lossless(cuda, mode, form):
    from edrixs_b200 import device
    ref, gpu = _ham(mode)
    P = device.pack(gpu, form=form)
    assert P is not None and 0 < P.vals.numel() <= device.PACK_VALUES_MAX
    assert P.wide == (form == "wide")
    _assert_pack_lossless(P, gpu)


def test_pack_refuses_too_many_values(cuda):
    import torch
    from edrixs_b200 import device
    rng = np.random.default_rng(0)
    n = 100
    M = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))  # 9900 distinct off-diagonal values
    A = device.CSR(torch.arange(0, n * n + 1, n, dtype=torch.int64, device="cuda"),
                   torch.arange(n, dtype=torch.int32, device="cuda").repeat(n),
                   torch.from_numpy(M.reshape(-1)).cuda(), n)
    assert device.pack(A) is None


def test_pack_rows_without_diagonal(cuda):
    """A matrix with an empty row and rows that have no diagonal entry."""
    import torch
    from edrixs_b200 import device
    rp = torch.tensor([0, 2, 2, 5, 6], dtype=torch.int64, device="cuda")
    col = torch.tensor([1, 3, 0, 2, 3, 0], dtype=torch.int32, device="cuda")
    val = torch.tensor([1 + 1j, -2, 3j, 4, 1 + 1j, -0.0], dtype=torch.complex128, device="cuda")
    A = device.CSR(rp, col, val, 4)
    P = device.pack(A)
    _assert_pack_lossless(P, A)
    assert P.vals.numel() == 4  # 1+1j, -2, 3j, -0.0 (sign of zero kept)


@pytest.mark.parametrize("k", [1, 6, 40, 64])
def test_packed_krylov_matches_oracle(cuda, k):
    import torch
    from edrixs_b200 import device
    ref, gpu = _ham("ham_i")
    P = device.pack(gpu)
    rng = np.random.default_rng(k)
    maxn = 25
    V0 = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    Vt = torch.from_numpy(V0).cuda()
    p = device.krylov(gpu, Vt, maxn, apply=dict(packed=P))
    c = device.krylov(gpu, Vt, maxn)
    assert torch.equal(p.neff, c.neff)
    assert torch.allclose(p.alpha, c.alpha, rtol=1e-10, atol=1e-10)
    assert torch.allclose(p.beta, c.beta, rtol=1e-10, atol=1e-10)
    for j in sorted({0, k // 2, k - 1}):
        a, b, nrm, neff = orc.build_krylov(ref, V0[:, j], maxn)
        assert p.neff[j].item() == neff
        assert np.allclose(p.alpha[j].cpu().numpy()[:neff], a, rtol=1e-8, atol=1e-8)
        assert np.allclose(p.beta[j].cpu().numpy()[:neff], b, rtol=1e-8, atol=1e-8)


@pytest.mark.parametrize("shape", [dict(col_group=6, threads=1024, blocks_per_sm=1, chunked=0),
                                   dict(col_group=8, threads=256, blocks_per_sm=4, chunked=1),
                                   dict(col_group=32, tiles=2, threads=1024, blocks_per_sm=1, chunked=0),
                                   dict(col_group=16, tiles=4, threads=256, blocks_per_sm=8, chunked=1),
                                   dict(col_group=6, threads=1024, blocks_per_sm=1, rowslot=1),
                                   dict(col_group=8, threads=256, blocks_per_sm=4, rowslot=1)])
def test_packed_launch_shapes_agree(cuda, shape):
    import torch
    from edrixs_b200 import device
    ref, gpu = _ham("ham_n")
    P = device.pack(gpu)
    k = 6 if shape["col_group"] <= 8 else 100
    rng = np.random.default_rng(4)
    V0 = torch.from_numpy(rng.normal(size=(gpu.nrows, k)) + 1j * rng.normal(size=(gpu.nrows, k))).cuda()
    p = device.krylov(gpu, V0, 20, apply=dict(shape, packed=P))
    c = device.krylov(gpu, V0, 20)
    assert torch.allclose(p.alpha, c.alpha, rtol=1e-10, atol=1e-10)
    assert torch.allclose(p.beta, c.beta, rtol=1e-10, atol=1e-10)


def test_packed_krylov_shifts_and_projections(cuda):
    import torch
    from edrixs_b200 import device
    ref, gpu = _ham("ham_i")
    P = device.pack(gpu)
    rng = np.random.default_rng(9)
    k, maxn = 3, 60
    V0 = torch.from_numpy(rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))).cuda()
    shifts = (np.array([0, 1, 2, 2]), np.array([-30 + 0.5j, -28 + 1j, -31 + 0.3j, -25 + 2j]))
    a = device.krylov(gpu, V0, maxn, proj=[gpu], shifts=shifts)
    b = device.krylov(gpu, V0, maxn, proj=[gpu], shifts=shifts, apply=dict(packed=P))
    assert torch.equal(a.shift_iters, b.shift_iters)
    assert torch.allclose(a.shift_y, b.shift_y, rtol=1e-9, atol=1e-12)
    assert torch.allclose(a.proj[0], b.proj[0], rtol=1e-9, atol=1e-9)


def _random_packable(n, per_row, nval, seed):
    """n x n complex128 CSR with per_row distinct random columns per row (the diagonal among
    them in some rows) and values drawn from nval distinct numbers."""
    import torch
    from edrixs_b200 import device
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    cols = torch.randint(0, n, (n, per_row), device="cuda", generator=g)
    cols[::3, 0] = torch.arange(0, n, 3, device="cuda")  # a diagonal entry in every third row
    cols, _ = torch.sort(cols, dim=1)
    keep = torch.ones_like(cols, dtype=torch.bool)
    keep[:, 1:] = cols[:, 1:] != cols[:, :-1]
    counts = keep.sum(dim=1)
    rp = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    rp[1:] = torch.cumsum(counts, 0)
    col = cols[keep].to(torch.int32)
    table = torch.complex(torch.randn(nval, device="cuda", dtype=torch.float64, generator=g),
                          torch.randn(nval, device="cuda", dtype=torch.float64, generator=g))
    val = table[torch.randint(0, nval, (col.numel(),), device="cuda", generator=g)]
    return device.CSR(rp, col, val, n)


def test_pack_wide_when_columns_leave_no_room(cuda):
    """2^24 + 1 columns leave 7 bits of the 32-bit word: 300 distinct values need the wide
    form.  "narrow" is refused, "auto" picks wide, and both products match the CSR's."""
    import torch
    from edrixs_b200 import device
    A = _random_packable((1 << 24) + 1, 2, 300, seed=3)
    assert device.pack(A, form="narrow") is None
    P = device.pack(A)
    assert P is not None and P.wide and P.vals.numel() == 300
    _assert_pack_lossless(P, A)
    rng = np.random.default_rng(1)
    X = torch.from_numpy(rng.normal(size=(A.nrows, 3)) + 1j * rng.normal(size=(A.nrows, 3))).cuda()
    ref = device.spmm(A, X)
    got = device.spmm(P, X)
    assert torch.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_pack_count_in_chunks(cuda):
    """More off-diagonal entries than one sort chunk (2^26): the count pass merges the chunks'
    value tables."""
    from edrixs_b200 import device
    A = _random_packable(1_500_000, 48, 1000, seed=11)
    assert A.nnz > (1 << 26) + 1_500_000
    P = device.pack(A)  # 21 column bits leave 11 for the 1000 values: the narrow form
    assert P is not None and not P.wide and P.vals.numel() == 1000
    _assert_pack_lossless(P, A)


@pytest.mark.parametrize("form", ["narrow", "wide"])
@pytest.mark.parametrize("k", [1, 3, 6, 40])
def test_spmm_packed_matches_csr(cuda, form, k):
    import torch
    from edrixs_b200 import device
    ref, gpu = _ham("ham_n")
    P = device.pack(gpu, form=form)
    rng = np.random.default_rng(k)
    X = torch.from_numpy(rng.normal(size=(gpu.nrows, k)) + 1j * rng.normal(size=(gpu.nrows, k))).cuda()
    Y0 = torch.from_numpy(rng.normal(size=(gpu.nrows, k)) + 1j * rng.normal(size=(gpu.nrows, k))).cuda()
    for al, sg, be in ((1.0, 0.0, 0.0), (-1.0, 2.5 + 0.5j, 0.0), (0.5j, 0.0, 1.0)):
        a = device.spmm(gpu, X, Y0.clone(), alpha=al, sigma=sg, beta=be)
        b = device.spmm(P, X, Y0.clone(), alpha=al, sigma=sg, beta=be)
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-12)
    # against the oracle's y += A x for one column
    x0 = X[:, 0].cpu().numpy()
    assert np.allclose(device.spmm(P, X[:, 0].contiguous()).cpu().numpy(), orc.matvec(ref, x0), rtol=1e-12,
                       atol=1e-12)


@pytest.mark.parametrize("k", [6, 64])
def test_wide_packed_krylov_matches_csr(cuda, k):
    """Lanczos on the wide form, with the packed matrix passed in place of the CSR."""
    import torch
    from edrixs_b200 import device
    ref, gpu = _ham("ham_n")
    P = device.pack(gpu, form="wide")
    rng = np.random.default_rng(k + 1)
    V0 = torch.from_numpy(rng.normal(size=(gpu.nrows, k)) + 1j * rng.normal(size=(gpu.nrows, k))).cuda()
    p = device.krylov(P, V0, 20)
    c = device.krylov(gpu, V0, 20)
    assert torch.equal(p.neff, c.neff)
    assert torch.allclose(p.alpha, c.alpha, rtol=1e-10, atol=1e-10)
    assert torch.allclose(p.beta, c.beta, rtol=1e-10, atol=1e-10)


def test_pack_diagonal_only_matrix(cuda):
    """No off-diagonal entries: an empty value table, and the product is the diagonal alone."""
    import torch
    from edrixs_b200 import device
    n = 1000
    d = torch.complex(torch.linspace(-1, 1, n, dtype=torch.float64), torch.linspace(0, 2, n, dtype=torch.float64))
    A = device.CSR(torch.arange(n + 1, dtype=torch.int64, device="cuda"),
                   torch.arange(n, dtype=torch.int32, device="cuda"), d.cuda(), n)
    P = device.pack(A)
    assert P is not None and P.nnz == 0 and P.vals.numel() == 0
    _assert_pack_lossless(P, A)
    X = torch.randn((n, 3), dtype=torch.float64, device="cuda").to(torch.complex128)
    assert torch.allclose(device.spmm(P, X), d.cuda()[:, None] * X, rtol=0, atol=1e-15)


@pytest.mark.parametrize("form", ["narrow", "wide"])
def test_rowslot_apply_matches_oracle(cuda, form):
    """One row per lane group (apply_rowslot) on both packed forms: Lanczos coefficients of
    the oracle to its tolerance, with shifts and projections as the batched RIXS runs them."""
    import torch
    from edrixs_b200 import device
    ref, gpu = _ham("ham_i")
    P = device.pack(gpu, form=form)
    rng = np.random.default_rng(12)
    k, maxn = 3, 40
    V0 = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    Vt = torch.from_numpy(V0).cuda()
    shifts = (np.array([0, 1, 2]), np.array([-30 + 0.5j, -28 + 1j, -31 + 0.3j]))
    a = device.krylov(gpu, Vt, maxn, proj=[gpu], shifts=shifts)
    b = device.krylov(gpu, Vt, maxn, proj=[gpu], shifts=shifts,
                      apply=dict(col_group=4, threads=256, blocks_per_sm=4, rowslot=1, packed=P))
    assert torch.equal(a.shift_iters, b.shift_iters)
    assert torch.allclose(a.alpha, b.alpha, rtol=1e-10, atol=1e-10)
    assert torch.allclose(a.shift_y, b.shift_y, rtol=1e-9, atol=1e-12)
    for j in range(k):  # the shifts stop the recurrence once they converge: compare that many steps
        n0 = b.neff[j].item()
        al, be, nrm, neff = orc.build_krylov(ref, V0[:, j], n0)
        assert neff == n0
        assert np.allclose(b.alpha[j].cpu().numpy()[:n0], al, rtol=1e-8, atol=1e-8)
        assert np.allclose(b.beta[j].cpu().numpy()[:n0], be, rtol=1e-8, atol=1e-8)
