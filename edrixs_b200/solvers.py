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
    may be a PackedMatrix when its CSR is no longer held, or a KronMatrix (the products run in
    its slab order; the eigenvectors are returned in the reference's row order)."""
    slab = isinstance(H, device.KronMatrix)
    if slab or isinstance(H, device.PackedMatrix):
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
        if not isinstance(H, device.CSR):
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
        # off-block-tridiagonal leakage after restarts is covered by using the full T.
        # Converged: residual <= tol x |Ritz value| (ARPACK's test, which this solver replaces
        # for ed_solver = 2), with |Ritz value| floored at 1
        conv = res[:want] <= tol * np.maximum(1.0, np.abs(theta[:want]))
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
    return theta[:nev].copy(), (H.from_slab(U).contiguous() if slab else U)


def _plain_replay(a, b, neff, computed, nev, max_niter, eval_tol):
    """The stopping logic of diag_ham_lanczos (src/lanczos.f90:76-131) replayed on Lanczos
    coefficients already computed: a[i-1] = alpha_i, b[i-1] = beta_i for i <= neff, where the
    device recurrence ran `computed` steps (neff < computed means beta_neff < 1e-10).  Every
    10th step and at max_niter the eigenvalues of T_i are taken (dsteqr, :169-206); once
    i >= nev the run stops when the nev-th one moved by less than eval_tol since the last
    check (the first check compares with 0).  Returns (evals[nev], ritz vectors of T_i, nkrylov),
    nkrylov = 0 when max_niter passes without convergence (the reference's eigenvectors are
    then zero), or None when more steps than were computed are needed."""
    from scipy.linalg import lapack

    def tri(i):
        d, z, info = lapack.dstev(np.asarray(a[:i], dtype=np.float64), np.asarray(b[:i - 1], dtype=np.float64),
                                  compute_v=1)
        if info != 0:
            raise RuntimeError(f"dstev info {info}")
        return np.concatenate([d, np.zeros(max(0, nev - i))]), z

    evals = np.zeros(nev)
    for i in range(1, max_niter + 1):
        if i > neff:
            return None  # the device recurrence has to run further
        if i % 10 == 0 or i == max_niter:
            ke, kv = tri(i)
            if i >= nev and abs(ke[nev - 1] - evals[nev - 1]) < eval_tol:
                return ke[:nev].copy(), kv, i
            evals = ke[:nev].copy()
        broke = neff < computed and i == neff
        if broke:  # beta_i < 1e-10: the Krylov space is exhausted
            if i >= 2:
                ke, kv = tri(i)
                evals = ke[:nev].copy()
            else:
                evals[0] = a[0]
                kv = np.ones((1, 1))
            return evals, kv, i
    return evals, None, 0


def plain_lanczos_eigs(H, nev, nvec, max_niter, eval_tol, seed=0, packed=None):
    """diag_ham_lanczos (src/lanczos.f90:6-167), the ed_solver = 1 path of
    src/ed_driver.f90:154-158, on the device.

    Plain Lanczos without reorthogonalisation, as the reference runs it: the start vector is
    uniform reals in [-0.5, 0.5), normalised (:60-70; seeded here, the reference's is not),
    and the coefficients come from libedx's recurrence (edx_krylov, one column, the
    reference's breakdown rule beta < 1e-10).  The stopping rule is replayed on them on the
    host (_plain_replay), running the device recurrence further (twice as many steps) until
    the rule decides.  Eigenvectors: the recurrence is run again for nkrylov steps and
    sum_i z_ij v_i accumulated on the device (:133-157), through an identity projection
    folded into accumulators.  On a degenerate spectrum the Krylov space holds one direction
    per distinct level, so the eigenvalues are the lowest distinct levels, as the reference
    reports them.  Returns (evals[nev] host array, evecs (n, nvec) device tensor)."""
    n = H.nrows
    rng = np.random.default_rng(seed)
    v1 = (rng.random(n) - 0.5).astype(np.complex128)
    v1 /= np.sqrt(np.vdot(v1, v1).real)
    V0 = torch.from_numpy(v1).to("cuda").reshape(-1, 1).contiguous()
    apply = dict(packed=packed) if packed is not None else None
    m = min(int(max_niter), 64)
    while True:
        r = device.krylov(H, V0, m, apply=apply)
        neff = int(r.neff[0].item())
        got = _plain_replay(r.alpha[0, :neff].cpu().numpy(), r.beta[0, :neff].cpu().numpy(), neff, m, nev,
                            int(max_niter), eval_tol)
        if got is not None:
            break
        m = min(int(max_niter), 2 * m)
    evals, kv, nk = got
    out = torch.zeros((n, nvec), dtype=torch.complex128, device="cuda")
    if nk > 0 and nvec > 0:
        q = min(nvec, kv.shape[1])
        coef = torch.zeros((nvec, nk), dtype=torch.complex128, device="cuda")
        coef[:q] = torch.from_numpy(np.ascontiguousarray(kv[:nk, :q].T)).to("cuda")
        eye = device.CSR(torch.arange(n + 1, dtype=torch.int64, device="cuda"),
                         torch.arange(n, dtype=torch.int32, device="cuda"),
                         torch.ones(n, dtype=torch.complex128, device="cuda"), n)
        device.krylov(H, V0, nk, proj=[eye], apply=apply,
                      accumulate=dict(window=min(8, nk), col=np.zeros(nvec, dtype=np.int32), coef=coef.contiguous(),
                                      out=[out]))
    return evals, out
