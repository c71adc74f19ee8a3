"""Parity of the CUDA kernels (through the C ABI) against the CPU oracle.

Bar: Fock basis, CSR row pointers, column indices and values bit-exact; SpMV/SpMM and the
Krylov / MINRES / continued-fraction / density-matrix results within the FP64 tolerances
stated per test.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu


def _model_terms(nbath, N, seed):
    from edrixs_b200 import siam
    m = siam.make_siam(nbath, N, seed)
    t = dict(
        hop_i=siam.text_roundtrip(siam.nonzero_terms(m.emat_i), 2),
        coul_i=siam.text_roundtrip(siam.nonzero_terms(m.umat_i), 4),
        hop_n=siam.text_roundtrip(siam.nonzero_terms(m.emat_n), 2),
        coul_n=siam.text_roundtrip(siam.nonzero_terms(m.umat_n), 4),
    )
    pin, pout = siam.rixs_polarisations()[1]
    t["tr_i"] = siam.text_roundtrip(siam.nonzero_terms(siam.polarised_operator(m, pin)), 2)
    t["tr_f"] = siam.text_roundtrip(siam.nonzero_terms(np.conj(siam.polarised_operator(m, pout)).T), 2)
    return m, t


def _to_np(csr):
    return (csr.row_ptr.cpu().numpy(), csr.col.cpu().numpy(), csr.val.cpu().numpy())


def _assert_bitexact(gpu, ref):
    rp, col, val = _to_np(gpu)
    assert np.array_equal(rp, ref.row_ptr)
    assert np.array_equal(col, ref.col)
    # values: identical summation order -> identical doubles
    assert np.array_equal(val.view(np.float64), ref.val.view(np.float64))


def test_fock_unrank_digests(cuda, golden_dir):
    from edrixs_b200 import device
    d = json.load(open(os.path.join(golden_dir, "fock_digests.json")))
    assert list(device.fock_unrank(4, 2).states.cpu().numpy()) == d["explicit_4_2"]
    for key in ("20_10", "20_11", "24_12", "26_13"):
        norb, N = map(int, key.split("_"))
        a = device.fock_unrank(norb, N).states.cpu().numpy().astype("<i8")
        assert hashlib.sha256(a.tobytes()).hexdigest() == d[key]["sha256"]


def test_basis_full_detection(cuda):
    from edrixs_b200 import device
    b = device.basis_from_states(orc.fock_full_N(12, 5))
    assert (b.norb, b.nelec) == (12, 5)
    sub = orc.fock_full_N(12, 5)[::3]
    assert device.basis_from_states(sub).norb == 0


@pytest.mark.parametrize("nbath,N", [(2, 3), (6, 8)])
def test_build_bitexact_all_modes(cuda, nbath, N):
    from edrixs_b200 import device
    m, t = _model_terms(nbath, N, seed=5)
    nv = m.nv
    fi, fn = orc.fock_full_N(nv, N), orc.fock_full_N(nv, N + 1)
    bi, bn = device.basis_from_states(fi), device.basis_from_states(fn)
    assert bi.norb == nv and bn.norb == nv
    ref = orc.build_csr("ham_i", fi, t["hop_i"], t["coul_i"], num_val_orbs=nv)
    _assert_bitexact(device.build_csr(device.HAM_I, bi, t["hop_i"], t["coul_i"], num_val_orbs=nv), ref)
    ref = orc.build_csr("ham_n", fn, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6)
    _assert_bitexact(device.build_csr(device.HAM_N, bn, t["hop_n"], t["coul_n"], num_val_orbs=nv,
                                      num_core_orbs=6), ref)
    z = 7.5 + 0.6j
    ref = orc.build_csr("ham_n", fn, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6, ham_sign=-1.0,
                        omega=z)
    _assert_bitexact(device.build_csr(device.HAM_N, bn, t["hop_n"], t["coul_n"], num_val_orbs=nv, num_core_orbs=6,
                                      ham_sign=-1.0, omega=z), ref)
    ref = orc.build_csr("trans_i", fn, t["tr_i"], fock_right=fi, num_val_orbs=nv, num_core_orbs=6)
    _assert_bitexact(device.build_csr(device.TRANS_I, bn, t["tr_i"], right=bi, num_val_orbs=nv, num_core_orbs=6),
                     ref)
    ref = orc.build_csr("trans_f", fi, t["tr_f"], fock_right=fn, num_val_orbs=nv, num_core_orbs=6)
    _assert_bitexact(device.build_csr(device.TRANS_F, bi, t["tr_f"], right=bn, num_val_orbs=nv, num_core_orbs=6),
                     ref)


def test_build_binary_search_basis(cuda):
    """A basis that is not a full sector (every third state): lookups use binary search."""
    from edrixs_b200 import device
    m, t = _model_terms(2, 5, seed=9)
    nv = m.nv
    sub = orc.fock_full_N(nv, 5)[::3].copy()
    b = device.basis_from_states(sub)
    assert b.norb == 0
    ref = orc.build_csr("ham_i", sub, t["hop_i"], t["coul_i"], num_val_orbs=nv)
    _assert_bitexact(device.build_csr(device.HAM_I, b, t["hop_i"], t["coul_i"], num_val_orbs=nv), ref)


def test_build_known_answer_files(cuda, golden_dir):
    from edrixs_b200 import device, io
    d = os.path.join(golden_dir, "known_answer")
    fock = io.read_fock(os.path.join(d, "fock_i.in"))
    hop, coul = io.read_hopping(os.path.join(d, "hopping_i.in")), io.read_coulomb(os.path.join(d, "coulomb_i.in"))
    ref = orc.build_csr("ham_i", fock.astype(np.int64), hop, coul, num_val_orbs=20)
    _assert_bitexact(device.build_csr(device.HAM_I, device.basis_from_states(fock), hop, coul, num_val_orbs=20), ref)


@pytest.fixture(scope="module")
def hn_pair(cuda):
    from edrixs_b200 import device
    m, t = _model_terms(6, 8, seed=5)
    fn = orc.fock_full_N(m.nv, 9)
    ref = orc.build_csr("ham_n", fn, t["hop_n"], t["coul_n"], num_val_orbs=m.nv, num_core_orbs=6)
    gpu = device.build_csr(device.HAM_N, device.basis_from_states(fn), t["hop_n"], t["coul_n"], num_val_orbs=m.nv,
                           num_core_orbs=6, want_c64=True)
    return ref, gpu


@pytest.mark.parametrize("k", [1, 3, 6, 8, 16, 40])
def test_spmm_c128(hn_pair, k):
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(k)
    X = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    Y0 = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    Xt = torch.from_numpy(X).cuda()
    Yt = torch.from_numpy(Y0).cuda()
    device.spmm(gpu, Xt, Yt, alpha=1.0, beta=1.0)  # y += A x
    want = np.stack([orc.matvec(ref, X[:, c], Y0[:, c].copy()) for c in range(k)], axis=1)
    got = Yt.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    # shifted form: y = z x - A x
    z = 2.0 - 0.5j
    Yt2 = device.spmm(gpu, Xt, alpha=-1.0, sigma=z)
    want2 = z * X - np.stack([orc.matvec(ref, X[:, c]) for c in range(k)], axis=1)
    assert np.abs(Yt2.cpu().numpy() - want2).max() <= 1e-13 * np.abs(want2).max()


@pytest.mark.parametrize("k", [1, 6, 8, 40])
def test_spmm_short_rows(cuda, k):
    """A transition operator (about 10 entries per row) takes the row-per-slot mapping."""
    import torch
    from edrixs_b200 import device
    m, t = _model_terms(6, 8, seed=5)
    fi, fn = orc.fock_full_N(m.nv, 8), orc.fock_full_N(m.nv, 9)
    ref = orc.build_csr("trans_f", fi, t["tr_f"], fock_right=fn, num_val_orbs=m.nv, num_core_orbs=6)
    gpu = device.build_csr(device.TRANS_F, device.basis_from_states(fi), t["tr_f"],
                           right=device.basis_from_states(fn), num_val_orbs=m.nv, num_core_orbs=6)
    assert ref.nnz <= 16 * ref.nrows
    rng = np.random.default_rng(k)
    X = rng.normal(size=(ref.ncols, k)) + 1j * rng.normal(size=(ref.ncols, k))
    Y0 = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    Yt = torch.from_numpy(Y0).cuda()
    device.spmm(gpu, torch.from_numpy(X).cuda(), Yt, alpha=1.0, beta=1.0)
    want = np.stack([orc.matvec(ref, X[:, c], Y0[:, c].copy()) for c in range(k)], axis=1)
    assert np.abs(Yt.cpu().numpy() - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("k", [1, 2])
def test_spmm_column_major_slices(hn_pair, k):
    """X given as a column slice of a column-major block (what an eigensolver returns): one
    column is used as is, wider slices are copied to row-major."""
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(3)
    B = rng.normal(size=(ref.nrows, 4)) + 1j * rng.normal(size=(ref.nrows, 4))
    Bt = torch.from_numpy(B).cuda().T.contiguous().T
    assert Bt.stride() == (1, ref.nrows)
    Y = device.spmm(gpu, Bt[:, :k].contiguous())
    want = np.stack([orc.matvec(ref, B[:, c]) for c in range(k)], axis=1)
    assert np.abs(Y.cpu().numpy() - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("k", [1, 8])
def test_spmm_c64(hn_pair, k):
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(k)
    X = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    want = np.stack([orc.matvec(ref, X[:, c]) for c in range(k)], axis=1)
    # complex64 matrix, complex128 vectors (FP64 accumulation)
    y = device.spmm(gpu, torch.from_numpy(X).cuda(), c64=True).cpu().numpy()
    assert np.abs(y - want).max() <= 2e-7 * np.abs(want).max()
    # complex64 matrix and vectors
    y = device.spmm(gpu, torch.from_numpy(X.astype(np.complex64)).cuda(), c64=True).cpu().numpy()
    assert np.abs(y - want).max() <= 2e-6 * np.abs(want).max()


def test_krylov_matches_oracle(hn_pair):
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(1)
    k, maxn = 3, 25
    V0 = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    res = device.krylov(gpu, torch.from_numpy(V0).cuda(), maxn)
    for c in range(k):
        a, b, nrm, neff = orc.build_krylov(ref, V0[:, c], maxn)
        assert res.neff[c].item() == neff
        assert abs(res.norm[c].item() - nrm) <= 1e-12 * nrm
        assert np.allclose(res.alpha[c].cpu().numpy()[:neff], a, rtol=1e-8, atol=1e-8)
        assert np.allclose(res.beta[c].cpu().numpy()[:neff], b, rtol=1e-8, atol=1e-8)


def test_krylov_start_columns_of_a_wider_block(hn_pair):
    """Start vectors given as a column slice of a wider row-major block (leading dimension >
    k) give the same recurrences as the same columns copied out."""
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(2)
    W = torch.from_numpy(rng.normal(size=(gpu.nrows, 7)) + 1j * rng.normal(size=(gpu.nrows, 7))).cuda()
    for s, e in ((2, 5), (6, 7)):
        a = device.krylov(gpu, W[:, s:e], 20)
        b = device.krylov(gpu, W[:, s:e].contiguous(), 20)
        assert torch.equal(a.alpha, b.alpha) and torch.equal(a.beta, b.beta) and torch.equal(a.norm, b.norm)


def test_krylov_early_stop(cuda, golden_dir):
    """A 45-dimensional space exhausts before maxn: beta < 1e-10 stops the column (:291)."""
    import torch
    from edrixs_b200 import device, io
    d = os.path.join(golden_dir, "known_answer")
    fock = io.read_fock(os.path.join(d, "fock_i.in"))
    hop, coul = io.read_hopping(os.path.join(d, "hopping_i.in")), io.read_coulomb(os.path.join(d, "coulomb_i.in"))
    ref = orc.build_csr("ham_i", fock.astype(np.int64), hop, coul, num_val_orbs=20)
    gpu = device.build_csr(device.HAM_I, device.basis_from_states(fock), hop, coul, num_val_orbs=20)
    v = np.ones(45, dtype=complex)
    a, b, nrm, neff = orc.build_krylov(ref, v, 200)
    r = device.krylov(gpu, torch.from_numpy(np.stack([v, v], 1)).cuda(), 200)
    assert neff < 200
    assert abs(r.neff[0].item() - neff) <= 1  # the exact stopping step is a rounding-level decision


def test_minres_matches_oracle(hn_pair):
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(2)
    b = rng.normal(size=ref.nrows) + 1j * rng.normal(size=ref.nrows)
    z = 35.0 + 0.6j
    # explicit A = z - H (the reference's matrix) on the oracle side
    x_ref, it_ref, res_ref = orc.minres(_shifted(ref, z), b, 1e-10, 3000)
    x, it, res = device.minres(gpu, torch.from_numpy(b).cuda(), 1e-10, 3000, alpha=-1.0, sigma=z)
    x = x.cpu().numpy()
    assert abs(it - it_ref) <= 2
    assert np.abs(x - x_ref).max() <= 1e-8 * np.abs(x_ref).max()


def _shifted(ref, z):
    """Oracle CSR of z*I - H with the diagonal merged like build_ham_n(ham_sign=-1)."""
    import scipy.sparse as sp
    M = (z * sp.identity(ref.nrows, format="csr") - ref.to_scipy()).tocsr()
    M.sort_indices()
    return orc.CSR(M.indptr.astype(np.int64), M.indices.astype(np.int32), M.data.astype(np.complex128), ref.ncols)


def test_multishift_equals_per_shift_minres(hn_pair):
    """All shifts of one seed from one Krylov space == separate MINRES runs (linsys.f90)."""
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(3)
    k = 2
    B = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    zs = [30.0 + 0.6j, 34.0 + 0.6j, 40.0 + 0.6j]
    scol = [c for c in range(k) for _ in zs]
    sz = [z for _ in range(k) for z in zs]
    maxn = 800
    # store the Lanczos vectors through an identity projector to rebuild x
    import scipy.sparse as sp
    from edrixs_b200.device import CSR
    I = sp.identity(ref.nrows, format="csr", dtype=np.complex128)
    eye = CSR(torch.from_numpy(I.indptr.astype(np.int64)).cuda(), torch.from_numpy(I.indices.astype(np.int32)).cuda(),
              torch.from_numpy(I.data).cuda(), ref.nrows)
    r = device.krylov(gpu, torch.from_numpy(B).cuda(), maxn, proj=[eye], shifts=(scol, sz), shift_tol=1e-10,
                      shift_maxit=maxn)
    V = r.proj[0].cpu().numpy()  # (k, steps + 1, n): the vectors the recurrence produced
    Y = r.shift_y.cpu().numpy()
    assert not Y[:, V.shape[1]:].any()
    for s in range(len(sz)):
        x = Y[s, :V.shape[1]] @ V[scol[s]]
        x_ref, it_ref, _ = orc.minres(_shifted(ref, sz[s]), B[:, scol[s]], 1e-10, maxn)
        assert abs(int(r.shift_iters[s]) - it_ref) <= 3
        assert np.abs(x - x_ref).max() <= 1e-7 * np.abs(x_ref).max()


def test_cf_spectrum_matches_golden(cuda, golden_dir):
    import torch
    from edrixs_b200 import device
    with np.load(os.path.join(golden_dir, "spectra.npz")) as z:
        g = {k: z[k] for k in z.files}
    dev = dict(device="cuda")
    w = orc.boltz_dist(g["eigval"], 10.0)
    s = device.cf_spectrum(torch.tensor(g["npoles"], dtype=torch.int32, **dev), torch.tensor(g["alpha"], **dev),
                           torch.tensor(g["beta"], **dev), g["eigval"], g["norm"], w, g["om_rixs"], g["gam_rixs"])
    assert np.abs(s.cpu().numpy() - g["s_rixs"]).max() <= 1e-10 * np.abs(g["s_rixs"]).max()


def test_denmat_matches_oracle(cuda, dense_small):
    import torch
    from edrixs_b200 import device
    g = dense_small
    nv = int(g["nv"])
    H = orc.build_csr("ham_i", g["fock_i"], (g["hop_i_idx"], g["hop_i_val"]), (g["coul_i_idx"], g["coul_i_val"]),
                      num_val_orbs=nv)
    e, v = np.linalg.eigh(H.dense())
    vecs = np.ascontiguousarray(v[:, :3])
    b = device.basis_from_states(g["fock_i"])
    got = device.denmat(b, nv, torch.from_numpy(vecs).cuda()).cpu().numpy()
    for c in range(3):
        want = orc.denmat(g["fock_i"], nv, vecs[:, c])
        assert np.abs(got[c] - want).max() < 1e-12


@pytest.mark.parametrize("c64", [False, True])
def test_krylov_csr_rowslot_matches(hn_pair, c64):
    """One row per lane group on the CSR (apply_rowslot): the same recurrences as the warp-per-
    row product, complex128 and complex64 matrices."""
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    if c64:
        gpu.to_c64()
    rng = np.random.default_rng(21)
    V0 = torch.from_numpy(rng.normal(size=(gpu.nrows, 6)) + 1j * rng.normal(size=(gpu.nrows, 6))).cuda()
    a = device.krylov(gpu, V0, 25, c64=c64)
    for shape in (dict(col_group=6, threads=256, blocks_per_sm=4, rowslot=1),
                  dict(col_group=8, threads=1024, blocks_per_sm=1, rowslot=1)):
        b = device.krylov(gpu, V0, 25, c64=c64, apply=shape)
        assert torch.equal(a.neff, b.neff)
        tol = 1e-6 if c64 else 1e-10
        assert torch.allclose(a.alpha, b.alpha, rtol=tol, atol=tol)
        assert torch.allclose(a.beta, b.beta, rtol=tol, atol=tol)
    if not c64:
        al, be, nrm, neff = orc.build_krylov(ref, V0[:, 0].cpu().numpy(), 25)
        assert np.allclose(b.alpha[0].cpu().numpy()[:neff], al, rtol=1e-8, atol=1e-8)


def test_krylov_zero_start_column(hn_pair):
    """A zero start vector among others: its recurrence stops after one step with norm 0 and
    finite coefficients (so it adds nothing to a spectrum), and the other columns are the
    same as without it."""
    import torch
    from edrixs_b200 import device
    ref, gpu = hn_pair
    rng = np.random.default_rng(31)
    V = rng.normal(size=(gpu.nrows, 3)) + 1j * rng.normal(size=(gpu.nrows, 3))
    V[:, 1] = 0
    r = device.krylov(gpu, torch.from_numpy(V).cuda(), 20)
    assert r.norm[1].item() == 0.0 and r.neff[1].item() == 1
    assert torch.isfinite(r.alpha).all() and torch.isfinite(r.beta).all()
    s = device.krylov(gpu, torch.from_numpy(V[:, [0, 2]].copy()).cuda(), 20)
    assert torch.allclose(r.alpha[[0, 2]], s.alpha, rtol=1e-12, atol=1e-12)
    spec = device.cf_spectrum(r.neff, r.alpha, r.beta, np.zeros(3), r.norm.cpu().numpy(), np.ones(3),
                              np.linspace(-5, 5, 50), 0.3, per_set=True)
    assert torch.isfinite(spec).all() and spec[1].abs().max().item() == 0.0


@pytest.mark.parametrize("nrows,k,maxn,m,nw,np_", [(1000, 3, 37, 29, 70, 2), (64, 1, 8, 8, 64, 1), (4097, 6, 50, 1, 5, 2)])
def test_proj_combine_equals_matmul(cuda, nrows, k, maxn, m, nw, np_):
    """edx_proj_combine (the batched RIXS's final-state start vectors from stored projections)
    equals the product and transpose it replaces, for ragged tiles of rows, shifts and
    Lanczos vectors."""
    import torch
    from edrixs_b200 import device
    g = torch.Generator(device="cuda")
    g.manual_seed(nrows + m)

    def rnd(*shape):
        return torch.complex(torch.randn(shape, dtype=torch.float64, device="cuda", generator=g),
                             torch.randn(shape, dtype=torch.float64, device="cuda", generator=g))

    projs = [rnd(k, maxn, nrows)[:, :m + (maxn - m) // 2, :] for _ in range(np_)]  # views, as krylov returns
    y = rnd(k * nw, maxn)
    got = device.proj_combine(projs, y, k, nw, m)
    Y = y.view(k, nw, maxn)[:, :, :m]
    want = torch.stack([torch.matmul(Y, P[:, :m, :]) for P in projs], dim=0).reshape(np_ * k * nw, nrows).T
    assert got.shape == want.shape
    assert float((got - want).abs().max()) <= 1e-13 * float(want.abs().max())
