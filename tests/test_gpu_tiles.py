"""The tiled layout (edx_tiles_*) and the tiled Lanczos product that runs on it.

Bar: the layout holds exactly the CSR's entries (same columns, bit-identical values, per row
in ascending column order); the Lanczos coefficients on the tiled product match the oracle
to the same FP64 tolerance as the CSR product (rtol 1e-8) and the CSR product itself to
1e-10 relative.
"""
import numpy as np
import pytest

from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu


def _hf(nbath=6, N=8, seed=5):
    from edrixs_b200 import device, siam
    m = siam.make_siam(nbath, N, seed)
    hop = siam.text_roundtrip(siam.nonzero_terms(m.emat_i), 2)
    coul = siam.text_roundtrip(siam.nonzero_terms(m.umat_i), 4)
    nv = m.nv
    ref = orc.build_csr("ham_i", orc.fock_full_N(nv, N), hop, coul, num_val_orbs=nv)
    basis = device.fock_unrank(nv, N)
    gpu = device.build_csr(device.HAM_I, basis, hop, coul, num_val_orbs=nv)
    return ref, gpu, basis


def _layout_to_rows(L):
    """Rebuild {row: [(col, value)...]} from the device arrays of a layout."""
    tr, tc = L.tile_r.cpu().numpy(), L.tile_c.cpu().numpy()
    pp, pc, prow = L.piece_ptr.cpu().numpy(), L.piece_ctile.cpu().numpy(), L.piece_rows.cpu().numpy()
    pe, ph = L.piece_ent.cpu().numpy(), L.piece_hdr.cpu().numpy()
    hdr = L.hdr.cpu().numpy().view(np.uint16)
    lcol, val = L.lcol.cpu().numpy(), L.val.cpu().numpy()
    rows = {}
    for R in range(len(tr) - 1):
        for p in range(pp[R], pp[R + 1]):
            ra, rb = prow[p] & 0xFFFF, prow[p] >> 16
            assert 0 <= ra < rb <= tr[R + 1] - tr[R]
            assert pe[p] % 16 == 0 and ph[p] % 8 == 0
            assert pe[p + 1] - pe[p] <= 1024
            for i in range(rb - ra):
                a, b = hdr[ph[p] + i], hdr[ph[p] + i + 1]
                for e in range(pe[p] + a, pe[p] + b):
                    rows.setdefault(tr[R] + ra + i, []).append((tc[pc[p]] + lcol[e], val[e]))
    return rows


def _assert_layout_equals_csr(L, gpu):
    rp, col, val = (gpu.row_ptr.cpu().numpy(), gpu.col.cpu().numpy(), gpu.val.cpu().numpy())
    rows = _layout_to_rows(L)
    assert sum(len(v) for v in rows.values()) == len(col)
    for r in range(len(rp) - 1):
        got = rows.get(r, [])
        want_c, want_v = col[rp[r]:rp[r + 1]], val[rp[r]:rp[r + 1]]
        assert [c for c, _ in got] == list(want_c), r
        assert np.array_equal(np.array([v for _, v in got], dtype=np.complex128).view(np.float64),
                              want_v.view(np.float64)), r


def test_fock_tiles_share_high_bits(cuda):
    from edrixs_b200 import device
    b = device.fock_unrank(16, 8)
    for m in (device.TILE_ROWS_MAX, device.TILE_COLS_MAX):
        t = device.fock_tiles(b.states, m).cpu().numpy()
        s = b.states.cpu().numpy().astype(np.uint64)
        assert t[0] == 0 and t[-1] == len(s) and np.all(np.diff(t) >= 1) and np.diff(t).max() <= m
        # one shift separates the tiles: states inside a tile share it, neighbours differ
        p = next(q for q in range(64) if all(len(set((s[a:c] >> np.uint64(q)).tolist())) == 1
                                             for a, c in zip(t[:-1], t[1:])))
        assert all((s[c - 1] >> np.uint64(p)) != (s[c] >> np.uint64(p)) for c in t[1:-1])


def test_layout_holds_the_csr(cuda):
    from edrixs_b200 import device
    ref, gpu, basis = _hf()
    L = device.tiles_for(gpu, basis)
    _assert_layout_equals_csr(L, gpu)


def test_layout_splits_large_pairs(cuda):
    """A dense 300 x 300 block: every (row tile, column tile) pair has more entries than one
    piece holds, so pairs are cut at row boundaries."""
    import torch
    from edrixs_b200 import device
    rng = np.random.default_rng(3)
    n = 300
    M = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    M = M + M.conj().T
    rp = torch.arange(0, n * n + 1, n, dtype=torch.int64, device="cuda")
    col = torch.arange(n, dtype=torch.int32, device="cuda").repeat(n)
    A = device.CSR(rp, col, torch.from_numpy(M.reshape(-1)).cuda(), n)
    tr = torch.tensor([0, 256, 300], dtype=torch.int32)
    tc = torch.tensor([0, 100, 200, 300], dtype=torch.int32)
    L = device.build_tiles(A, tr, tc)
    assert L.npiece > 6
    _assert_layout_equals_csr(L, A)
    V0 = torch.from_numpy(rng.normal(size=(n, 40)) + 1j * rng.normal(size=(n, 40))).cuda()
    a = device.krylov(A, V0, 30)
    b = device.krylov(A, V0, 30, apply=dict(layout=L))
    assert torch.allclose(a.alpha, b.alpha, rtol=1e-10, atol=1e-10)
    assert torch.allclose(a.beta, b.beta, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("k", [1, 40, 64])
def test_tiled_krylov_matches_oracle(cuda, k):
    import torch
    from edrixs_b200 import device
    ref, gpu, basis = _hf()
    L = device.tiles_for(gpu, basis)
    rng = np.random.default_rng(k)
    maxn = 25
    V0 = rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))
    Vt = torch.from_numpy(V0).cuda()
    t = device.krylov(gpu, Vt, maxn, apply=dict(layout=L))
    c = device.krylov(gpu, Vt, maxn)
    assert torch.equal(t.neff, c.neff)
    assert torch.allclose(t.alpha, c.alpha, rtol=1e-10, atol=1e-10)
    assert torch.allclose(t.beta, c.beta, rtol=1e-10, atol=1e-10)
    for j in sorted({0, k // 2, k - 1}):
        a, b, nrm, neff = orc.build_krylov(ref, V0[:, j], maxn)
        assert t.neff[j].item() == neff
        assert np.allclose(t.alpha[j].cpu().numpy()[:neff], a, rtol=1e-8, atol=1e-8)
        assert np.allclose(t.beta[j].cpu().numpy()[:neff], b, rtol=1e-8, atol=1e-8)


def test_tiled_krylov_shifts_and_projections(cuda):
    """The shifted-MINRES coefficients and the projections ride on the tiled product too."""
    import torch
    from edrixs_b200 import device
    ref, gpu, basis = _hf()
    L = device.tiles_for(gpu, basis)
    rng = np.random.default_rng(9)
    k, maxn = 3, 60
    V0 = torch.from_numpy(rng.normal(size=(ref.nrows, k)) + 1j * rng.normal(size=(ref.nrows, k))).cuda()
    shifts = (np.array([0, 1, 2, 2]), np.array([-30 + 0.5j, -28 + 1j, -31 + 0.3j, -25 + 2j]))
    a = device.krylov(gpu, V0, maxn, proj=[gpu], shifts=shifts)
    b = device.krylov(gpu, V0, maxn, proj=[gpu], shifts=shifts, apply=dict(layout=L))
    assert torch.equal(a.shift_iters, b.shift_iters)
    assert torch.allclose(a.shift_y, b.shift_y, rtol=1e-9, atol=1e-12)
    assert torch.allclose(a.proj[0], b.proj[0], rtol=1e-9, atol=1e-9)


def test_tiles_reject_bad_tiles(cuda):
    import torch
    from edrixs_b200 import device
    from edrixs_b200._lib import EdxError
    ref, gpu, basis = _hf()
    n = gpu.nrows
    with pytest.raises(EdxError, match="tile"):
        device.build_tiles(gpu, torch.tensor([0, n], dtype=torch.int32), device.fock_tiles(basis.states, 128))
    with pytest.raises(EdxError, match="end at"):
        device.build_tiles(gpu, torch.tensor([0, 5], dtype=torch.int32), torch.tensor([0, 5], dtype=torch.int32))
