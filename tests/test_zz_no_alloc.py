"""edx_denmat_static: the density matrix for callers that cannot allocate device memory.

Such callers (a host whose HBM is fully reserved by its own allocator, or a foreign-language
binding that only forwards the buffers it was given) cannot create the workspace that
edx_denmat takes, so this entry point keeps its partial sums in a fixed device array inside
the library.  The test calls both entry points through the C ABI on the same eigenvectors
and requires the same result, on two calls in a row (the second call reuses the array the
first one left behind).  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(nv=12, nelec=5, nvec=3, seed=0):
    import torch
    from edrixs_b200 import device, siam
    from oracle import pyoracle as orc
    m = siam.make_siam(nv - 10, nelec, seed)
    hop = siam.text_roundtrip(siam.nonzero_terms(m.emat_i), 2)
    coul = siam.text_roundtrip(siam.nonzero_terms(m.umat_i), 4)
    H = orc.build_csr("ham_i", orc.fock_full_N(nv, nelec), hop, coul, num_val_orbs=nv)
    e, v = np.linalg.eigh(H.dense())
    basis = device.fock_unrank(nv, nelec)
    vecs = torch.from_numpy(np.ascontiguousarray(v[:, :nvec])).cuda()
    return basis, vecs, nv, nvec


def test_denmat_static_matches_workspace_version(cuda):
    import torch
    from edrixs_b200 import _lib
    from edrixs_b200.device import _ptr, _stream, _work
    L = _lib.load()
    basis, vecs, nv, nvec = _setup()
    n = basis.ndim
    ref = torch.zeros((nvec, nv, nv), dtype=torch.complex128, device="cuda")
    ws = ctypes.c_size_t(0)
    assert L.edx_denmat_workspace(n, nv, nvec, ctypes.byref(ws)) == 0
    w = _work(ws.value)
    assert L.edx_denmat(_ptr(basis.states), n, basis.norb, basis.nelec, nv, nvec, _ptr(vecs), _ptr(ref), _ptr(w),
                        ws.value, _stream()) == 0
    want = ref.cpu().numpy()
    for call in range(2):
        out = torch.full((nvec, nv, nv), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
        rc = L.edx_denmat_static(_ptr(basis.states), n, basis.norb, basis.nelec, nv, nvec, _ptr(vecs), _ptr(out),
                                 _stream())
        assert rc == 0, L.edx_last_error()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        # same kernel; at this size both entry points use the same 4 row chunks
        assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max()), f"call {call}"
        tr = np.trace(got, axis1=1, axis2=2).real
        assert np.allclose(tr, 5.0, atol=1e-10)  # N electrons in every eigenvector


def _both(L, basis, vecs, nv, nvec):
    """edx_denmat (with a workspace) and edx_denmat_static on the same input."""
    import torch
    from edrixs_b200.device import _ptr, _stream, _work
    n = basis.ndim
    ref = torch.zeros((nvec, nv, nv), dtype=torch.complex128, device="cuda")
    ws = ctypes.c_size_t(0)
    assert L.edx_denmat_workspace(n, nv, nvec, ctypes.byref(ws)) == 0
    w = _work(ws.value)
    assert L.edx_denmat(_ptr(basis.states), n, basis.norb, basis.nelec, nv, nvec, _ptr(vecs), _ptr(ref), _ptr(w),
                        ws.value, _stream()) == 0
    outs = []
    for _ in range(2):
        out = torch.full((nvec, nv, nv), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
        rc = L.edx_denmat_static(_ptr(basis.states), n, basis.norb, basis.nelec, nv, nvec, _ptr(vecs), _ptr(out),
                                 _stream())
        assert rc == 0, L.edx_last_error()
        outs.append(out.cpu().numpy())
    return ref.cpu().numpy(), outs


def test_denmat_static_above_the_chunk_cap(cuda):
    """38,760 rows (20 orbitals, 6 electrons): edx_denmat splits them into more than the 64
    row chunks the static array holds, so edx_denmat_static takes the clamped path (64 longer
    chunks).  The two differ only in summation order."""
    import torch
    from edrixs_b200 import _lib, device
    L = _lib.load()
    nv, nelec, nvec = 20, 6, 3
    basis = device.fock_unrank(nv, nelec)
    assert basis.ndim > 64 * 256
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    v = torch.randn((basis.ndim, nvec), dtype=torch.float64, device="cuda", generator=g) + \
        1j * torch.randn((basis.ndim, nvec), dtype=torch.float64, device="cuda", generator=g)
    v = (v / torch.linalg.vector_norm(v, dim=0, keepdim=True)).contiguous()
    want, outs = _both(L, basis, v, nv, nvec)
    for call, got in enumerate(outs):
        assert np.all(np.isfinite(got))
        assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max()), f"call {call}"
        assert np.allclose(np.trace(got, axis1=1, axis2=2).real, nelec, atol=1e-10)


def test_denmat_static_rejects_oversize(cuda):
    import torch
    from edrixs_b200 import _lib
    from edrixs_b200.device import _ptr, _stream
    L = _lib.load()
    basis, vecs, nv, nvec = _setup()
    out = torch.zeros(1, dtype=torch.complex128, device="cuda")
    # 5 vectors x 30 x 30 orbitals = 4500 entries > the 4096-entry static limit
    rc = L.edx_denmat_static(_ptr(basis.states), basis.ndim, basis.norb, basis.nelec, 30, 5, _ptr(vecs), _ptr(out),
                             _stream())
    assert rc == 1  # EDX_ERR_INVALID
    assert b"static scratch limit" in L.edx_last_error()
