"""Ground-state eigensolver and Krylov drivers on the device.

``lowest_eigs`` replaces diag_ham_arpack (src/arpack.f90:2-112, pznaupd 'SR' + pzneupd)
and the plain Lanczos of diag_ham_lanczos (src/lanczos.f90:6-167) with a block
thick-restart Lanczos:

* the Krylov block is expanded by one SpMM of width b per step (libedx ``edx_spmm``, or
  ``edx_spmm_packed`` on the packed form of H);
* every new block is orthogonalised against the whole basis twice (classical Gram-Schmidt,
  CGS2): tall-skinny contractions C = V^H W and W -= V^T C that libedx runs as single
  bandwidth-bound passes over the basis (``edx_gs_dot`` / ``edx_gs_update``), then the
  block is factorised by CholeskyQR2;
* the projected matrix T = V^H H V is accumulated from those coefficients, so after a
  restart the kept Ritz vectors and their coupling to the residual block are exact;
* Ritz pairs are accepted when || H u - theta u || <= tol; the block size b >= the
  multiplicity of the wanted eigenvalues (Kramers pairs at odd N) finds all copies.

Dense problems below ``min_ndim`` (and ed_solver = 0) use a dense Hermitian eigensolver on
the device, as the reference switches to ZHEEV there (src/ed_driver.f90:65-72,127-152).
"""
import numpy as np
import torch

from . import device


def _qr(W):
    Q, R = torch.linalg.qr(W, mode="reduced")
    return Q, R


def _cholqr2(W, gram=None, rmul=None):
    """W = Q R for a tall-skinny block by CholeskyQR2 (Fukaya, Nakatsukasa, Yanagisawa,
    Yamamoto 2014): twice, R from the Cholesky factor of the small Gram matrix W^H W and
    Q = W R^-1.  Two passes over W instead of a Householder factorisation, which is slow for
    millions of rows and a few columns.  A block too ill-conditioned for it (a Krylov space
    about to break down) goes to Householder QR.  gram(Q) -> Q^H Q and rmul(Q, M): Q = Q M in
    place; libedx's single-pass kernels (edx_gs_gram / edx_gs_rmul) unless given.  Returns
    (Q, R) with R a host array (a device tensor on the Householder path)."""
    gram = gram or device.gs_gram
    rmul = rmul or device.gs_rmul
    k = W.shape[1]
    if k > 8:
        return _qr(W)
    Q = W.contiguous().clone()
    Rt = np.eye(k, dtype=np.complex128)
    for _ in range(2):
        G = gram(Q).cpu().numpy()
        G = 0.5 * (G + G.conj().T)
        try:
            L = np.linalg.cholesky(G)
        except np.linalg.LinAlgError:
            return _qr(W)
        R = L.conj().T
        d = np.abs(np.diag(R))
        if not np.all(np.isfinite(d)) or d.min() <= 1e-7 * d.max():
            return _qr(W)
        rmul(Q, np.linalg.inv(R))   # Q = Q R^-1 in place
        Rt = R @ Rt
    return Q, Rt


def dense_eigs(H: device.CSR, nev):
    n = H.nrows
    rows = torch.repeat_interleave(torch.arange(n, device=H.val.device), H.row_ptr[1:] - H.row_ptr[:-1])
    Hd = torch.zeros((n, H.ncols), dtype=H.val.dtype, device=H.val.device)
    Hd[rows, H.col.to(torch.int64)] = H.val
    e, v = torch.linalg.eigh(Hd)  # ZHEEV('V','U') of full_diag.f90 uses the upper triangle; H is Hermitian
    return e[:nev].cpu().numpy(), v[:, :nev].contiguous()


def lowest_eigs(H: device.CSR, nev, nvec=None, tol=1e-9, block=None, mmax=None, max_restarts=200, seed=20240917,
                c64=False, verbose=False, packed=None):
    """Lowest `nev` eigenvalues (ascending) and `nvec` eigenvectors (n, nvec) of Hermitian H.
    packed: the packed form of H (device.pack); the block products then run on it.  H itself
    may be a PackedMatrix when its CSR is no longer held."""
    if isinstance(H, device.PackedMatrix):
        packed = H
    n = H.nrows
    nvec = nev if nvec is None else nvec
    want = max(nev, nvec)
    b = block if block is not None else min(max(want, 2), 4)
    b = max(1, min(b, n))
    if mmax is None:
        mmax = max(3 * want + 4 * b, 40)
    mmax = ((mmax + b - 1) // b) * b
    if n <= max(mmax + b, 64):
        if isinstance(H, device.PackedMatrix):
            raise ValueError("lowest_eigs: the dense solver of a small matrix needs its CSR")
        return dense_eigs(H, nev)[0], dense_eigs(H, nvec)[1]
    dev = torch.device("cuda", torch.cuda.current_device())
    dt = torch.complex128
    V = torch.zeros((mmax + b, n), dtype=dt, device=dev)  # basis vectors as rows
    T = np.zeros((mmax + b, mmax + b), dtype=np.complex128)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    X0 = torch.randn((n, b), dtype=torch.float64, device=dev, generator=g) + \
        1j * torch.randn((n, b), dtype=torch.float64, device=dev, generator=g)
    Q, _ = _qr(X0.to(dt))
    V[:b] = Q.T
    j = 0          # start of the block to expand
    theta = None
    for restart in range(max_restarts):
        while j + b <= mmax:
            X = V[j:j + b].T.contiguous()
            W = (device.spmm(packed, X) if packed is not None else device.spmm(H, X, c64=c64)).contiguous()
            # classical Gram-Schmidt twice against the whole basis (libedx: one pass over V each)
            C = device.gs_dot(V, j + b, W)
            device.gs_update(V, j + b, W, C)
            C2 = device.gs_dot(V, j + b, W)
            device.gs_update(V, j + b, W, C2)
            C = C + C2
            Q, R = _cholqr2(W)
            V[j + b:j + 2 * b] = Q.T
            T[:j + b, j:j + b] = C.cpu().numpy()
            T[j + b:j + 2 * b, j:j + b] = R if isinstance(R, np.ndarray) else R.cpu().numpy()
            j += b
        m = mmax
        Tm = T[:m, :m]
        Th = 0.5 * (Tm + Tm.conj().T)
        theta, Y = np.linalg.eigh(Th)
        Bl = T[m:m + b, m - b:m]
        res = np.linalg.norm(Bl @ Y[m - b:m, :], axis=0)
        # off-block-tridiagonal leakage after restarts is covered by using the full T
        conv = res[:want] <= tol * max(1.0, 1.0)
        if verbose:
            print(f"restart {restart}: theta={theta[:want]} res={res[:want]}")
        if np.all(conv):
            break
        # thick restart: keep the lowest `keep` Ritz vectors + the residual block
        keep = min(m - b, max(want + b, (m // 2 // b) * b))
        Yk = torch.from_numpy(Y[:, :keep].copy()).to(dev)
        U = Yk.T @ V[:m]                       # keep x n
        R_last = V[m:m + b].clone()
        V.zero_()
        V[:keep] = U
        V[keep:keep + b] = R_last
        Tn = np.zeros_like(T)
        Tn[:keep, :keep] = np.diag(theta[:keep])
        cpl = Bl @ Y[m - b:m, :keep]           # b x keep
        Tn[keep:keep + b, :keep] = cpl
        Tn[:keep, keep:keep + b] = cpl.conj().T
        T = Tn
        j = keep
    else:
        raise RuntimeError(f"lowest_eigs: not converged after {max_restarts} restarts (res={res[:want]})")
    Yv = torch.from_numpy(Y[:, :nvec].copy()).to(dev)
    U = (Yv.T @ V[:m]).T.contiguous()          # n x nvec
    U = U / torch.linalg.vector_norm(U, dim=0, keepdim=True)
    return theta[:nev].copy(), U
