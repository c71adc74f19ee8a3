"""Impurity x bath ("slab") form of an impurity-model Hamiltonian, for the structured product.

The reference builds every Hamiltonian as a flat CSR (src/ham.f90:2-711) and multiplies it
row by row (src/spmv.f90:73-103).  In an impurity model the two-body terms touch only the
impurity orbitals (and, in the core-hole sector, the core orbitals); the bath orbitals carry
one-body terms only: their levels and the hybridisation with the impurity.  Write every Fock
state as (I, B): I the occupation of the "A" orbitals (impurity + core), B that of the bath.
Then H is a sum of three kinds of operators:

* A-terms (all indices in A): they change I only, so they act as H_A (x) 1 on the slab of I,
  the contiguous block of rows with that impurity configuration;
* bath levels n_b: diagonal, d_B(B);
* hybridisation c+_a c_b and c+_b c_a (a in A, b in the bath): they map slab I + a (or
  I - a) onto slab I, and inside the slab they are a fixed hop of one bath electron, whose
  target row is a table lookup.

The structured product (libedx ``k_lanczos_apply_kron``) therefore reads whole slabs, not
scattered rows: each output slab sums about (nnz of its H_A row + 2 x hybridising orbitals)
source slabs, staged in shared memory by the tensor-memory accelerator.  No matrix is
streamed at all; its "entries" are H_A (a few thousand rows), the bath tables and a
hybridisation table of at most 16 x 16 values.

Rows are reordered slab by slab (the slab order); the Lanczos coefficients do not depend on
the row order, and ``perm`` maps slab rows back to the reference's rows.  The form exists when:
the bath is a contiguous run of valence bits; every four-fermion term lies in A; every
hopping term that touches the bath is a bath level or an A-bath hop; every A-term has an even
number of operators above the bath (so that its sign does not depend on B); and the basis is
the full product of A configurations and bath sectors.  Otherwise ``kron_spec`` returns None
and the CSR / packed products are used.

Fermion signs follow src/fock.f90:38-68: an operator on orbital p contributes
(-1)^(occupied orbitals below p).  With B the bath bits [b0, b0 + nb) and A_lo / A_hi the A
orbitals below / above them, for a row (I', B') with m' bath electrons:
  c+_a c_b (b destroyed, a created; source (I' + a, B' - b)):
     sign = (-1)^(|I'_lo| + |I' below a| + [a in A_hi](m' - 1)) * (-1)^(|B' below b|)
  c+_b c_a (a destroyed, b created; source (I' - a, B' + b)):
     sign = (-1)^(|I' below a| + [a in A_hi] m' + |I'_lo| - [a in A_lo]) * (-1)^(|B' below b|)
where "below" counts set bits at lower positions in the compressed A (or bath) numbering.
"""
from dataclasses import dataclass
from math import comb

import numpy as np

KRON_NB_MAX = 16       # bath orbitals (uint16 bath tables)
KRON_NAH_MAX = 16      # hybridising A orbitals


def _popc_vec(x):
    """popcount of a uint64 array (vectorised)."""
    x = np.asarray(x, dtype=np.uint64).copy()
    c = np.zeros(x.shape, dtype=np.int64)
    while np.any(x):
        c += (x & np.uint64(1)).astype(np.int64)
        x >>= np.uint64(1)
    return c


def _colex(nb, m):
    """All nb-bit configurations with m bits set, ascending (the colex rank order)."""
    if m < 0 or m > nb:
        return np.zeros(0, dtype=np.int64)
    out = []
    # Gosper's hack over m-subsets of nb bits, ascending
    if m == 0:
        return np.zeros(1, dtype=np.int64)
    v = (1 << m) - 1
    lim = 1 << nb
    while v < lim:
        out.append(v)
        c = v & -v
        r = v + c
        v = (((r ^ v) >> 2) // c) | r
    return np.array(out, dtype=np.int64)


@dataclass
class KronSpec:
    """Host arrays of the slab form (see the module docstring); all indices 0-based."""
    n: int                 # rows
    nb: int                # bath orbitals
    b0: int                # first bath bit of the full state
    a_bits: np.ndarray     # int64[nA] full-state bit of each A orbital, ascending (compressed index = position)
    n_alo: int             # A orbitals below the bath
    slab_cfg: np.ndarray   # uint32[nslab] compressed A configuration
    slab_full: np.ndarray  # int64[nslab] A configuration as a full-state bit pattern
    slab_m: np.ndarray     # int32[nslab] bath electrons of the slab
    slab_off: np.ndarray   # int32[nslab + 1] first row of each slab
    hyb_a: np.ndarray      # int32[nah] compressed A index of each hybridising A orbital
    t_cre: np.ndarray      # complex128[nah, nb]: coefficient of c+_a c_b (bath b destroyed, a created)
    t_ann: np.ndarray      # complex128[nah, nb]: coefficient of c+_b c_a (a destroyed, bath b created)
    up: np.ndarray         # int32[nslab, nah] slab of I + hyb_a[q] (-1: none)
    dn: np.ndarray         # int32[nslab, nah] slab of I - hyb_a[q] (-1: none)
    b_off: np.ndarray      # int32[nb + 2] first table index of each bath sector
    b_cfg: np.ndarray      # uint16[2^nb] bath configurations, sector by sector, colex
    b_nbr: np.ndarray      # uint16[2^nb, nb] rank of cfg ^ (1 << x) in its sector
    b_diag: np.ndarray     # complex128[2^nb] bath-level energy of each configuration
    a_hop: tuple           # A-terms (idx, val) of the hopping list
    a_coul: tuple          # A-terms (idx, val) of the Coulomb list
    perm: object           # int64[n] reference row of each slab row (numpy, or a tensor on the basis's device)

    @property
    def nslab(self):
        return len(self.slab_m)

    @property
    def nah(self):
        return len(self.hyb_a)

    @property
    def max_rows(self):
        return int(np.diff(self.slab_off).max())


def _slab_perm_host(full, m, sizes, slab_off, b_cfg, b_off, b0, nv, kidx, basis):
    """Reference row of every slab row: slab s, rank r is the state with A bits full[s] and
    bath configuration b_cfg[b_off[m[s]] + r] at bit b0; its row is the valence state's index
    in the ascending basis (times the core-hole index k, k-major, when kidx is given).  None
    when a state is missing from the basis or two slab rows meet one reference row."""
    n_rows = int(slab_off[-1])
    srow = np.repeat(np.arange(len(full)), sizes)
    rank = np.arange(n_rows) - slab_off[srow]
    full_row = full[srow] | (b_cfg[b_off[m[srow]] + rank] << b0)
    val = full_row & ((1 << nv) - 1)
    vidx = np.searchsorted(basis, val)
    if np.any(vidx >= len(basis)) or np.any(basis[np.minimum(vidx, len(basis) - 1)] != val):
        return None
    perm = kidx[full_row >> nv] * len(basis) + vidx if kidx is not None else vidx
    if np.bincount(perm, minlength=n_rows).max() != 1:
        return None
    return perm


def _slab_perm_device(full, m, sizes, slab_off, b_cfg, b_off, b0, nv, kidx, basis):
    """_slab_perm_host on the basis tensor's device (tens of millions of rows in milliseconds
    instead of a minute on the host); returns a device int64 tensor."""
    import torch
    dev = basis.device

    def t(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=dev)

    n_rows = int(slab_off[-1])
    srow = torch.repeat_interleave(torch.arange(len(full), device=dev), t(sizes))
    rank = torch.arange(n_rows, device=dev) - t(slab_off)[srow]
    full_row = t(full)[srow] | (t(b_cfg)[t(b_off)[t(m)[srow]] + rank] << b0)
    del srow, rank
    val = full_row & ((1 << nv) - 1)
    vidx = torch.searchsorted(basis, val)
    if bool((vidx >= len(basis)).any()) or bool((basis[vidx.clamp(max=len(basis) - 1)] != val).any()):
        return None
    del val
    perm = t(kidx)[full_row >> nv] * len(basis) + vidx if kidx is not None else vidx
    del full_row
    if int(torch.bincount(perm, minlength=n_rows).max()) != 1:
        return None
    return perm


def kron_spec(hopping, coulomb, basis_states, mode="ham_i", num_val_orbs=0, num_core_orbs=0, min_nb=4):
    """The slab form of the Hamiltonian built from these terms over this basis, or None.

    hopping / coulomb: (idx int[n, 2 or 4] 1-based, val complex[n]) as read from the *.in files
    (src/io.f90:93-152); basis_states: the valence Fock basis of the matrix (ascending);
    mode: "ham_i" (rows = basis states) or "ham_n" (rows = core-hole configuration k x basis
    state, k-major, src/ham.f90:414-446, with num_core_orbs core orbitals above the valence).
    basis_states may be a device tensor (int64): the row permutation is then computed on its
    device and ``perm`` is a device tensor."""
    hi = np.asarray(hopping[0], dtype=np.int64).reshape(-1, 2) - 1 if hopping is not None else np.zeros((0, 2), int)
    hv = np.asarray(hopping[1], dtype=np.complex128).reshape(-1) if hopping is not None else np.zeros(0, complex)
    ci = np.asarray(coulomb[0], dtype=np.int64).reshape(-1, 4) - 1 if coulomb is not None else np.zeros((0, 4), int)
    cv = np.asarray(coulomb[1], dtype=np.complex128).reshape(-1) if coulomb is not None else np.zeros(0, complex)
    nv, nc = int(num_val_orbs), int(num_core_orbs)
    if mode not in ("ham_i", "ham_n"):
        return None
    if mode == "ham_i":
        nc = 0
    on_device = not isinstance(basis_states, np.ndarray) and hasattr(basis_states, "device")
    basis = basis_states if on_device else np.asarray(basis_states, dtype=np.int64)
    if nv <= 0 or len(basis) == 0:
        return None
    nval_e = bin(int(basis[0])).count("1")
    # bath: valence orbitals in no four-fermion term, one contiguous run
    in_coul = np.zeros(nv + nc, dtype=bool)
    in_coul[ci.ravel()] = True
    free = [p for p in range(nv) if not in_coul[p]]
    if len(free) < min_nb:
        return None
    runs, start = [], free[0]
    for a, b in zip(free, free[1:] + [None]):
        if b != a + 1:
            runs.append((start, a + 1))
            start = b
    b0, b1 = max(runs, key=lambda r: r[1] - r[0])
    nb = b1 - b0
    if nb < min_nb or nb > KRON_NB_MAX:
        return None
    in_b = lambda p: (p >= b0) & (p < b1)  # noqa: E731
    a_bits = np.array([p for p in range(nv + nc) if not (b0 <= p < b1)], dtype=np.int64)
    n_alo = int(np.sum(a_bits < b0))
    cidx = {int(p): i for i, p in enumerate(a_bits)}
    # classify the terms
    if np.any(in_b(ci)):
        return None
    hop_a = np.zeros(len(hi), dtype=bool)
    b_level = np.zeros(nb, dtype=np.complex128)
    hyb = []  # (kind, a_compressed, b_local, value) kind 0: c+_a c_b, 1: c+_b c_a
    for t, (al, be) in enumerate(hi):  # term applies c_al then c+_be (src/ham.f90:63-77)
        ba, bb = in_b(al), in_b(be)
        if not ba and not bb:
            hop_a[t] = True
        elif ba and bb:
            if al != be:
                return None  # off-diagonal bath hopping: not in this form
            b_level[al - b0] += hv[t]
        elif ba:  # destroy bath al, create A be
            hyb.append((0, cidx[int(be)], int(al - b0), hv[t]))
        else:     # destroy A al, create bath be
            hyb.append((1, cidx[int(al)], int(be - b0), hv[t]))
    # an A-term's sign must not depend on the bath: an even number of operators above it
    for idx in list(hi[hop_a]) + list(ci):
        if int(np.sum(np.asarray(idx) >= b1)) % 2:
            return None
    act = sorted({a for _, a, _, v in hyb})
    if any(a_bits[a] >= nv for a in act):
        return None  # a core orbital hybridising with the bath: its slabs would change the core count
    if len(act) > KRON_NAH_MAX:
        return None
    qof = {a: q for q, a in enumerate(act)}
    nah = len(act)
    t_cre = np.zeros((nah, nb), dtype=np.complex128)
    t_ann = np.zeros((nah, nb), dtype=np.complex128)
    for kind, a, b, v in hyb:
        (t_cre if kind == 0 else t_ann)[qof[a], b] += v
    # A configurations: valence part with 0..nb bath electrons left, core part with one hole
    nA = len(a_bits)
    nA_val = int(np.sum(a_bits < nv))
    if nA > 20:
        return None
    cfgs = np.arange(1 << nA, dtype=np.int64)
    val_mask_c = (1 << nA_val) - 1  # valence A orbitals come first in the compressed numbering
    nval_a = _popc_vec((cfgs & val_mask_c).astype(np.uint64))
    ncore = _popc_vec((cfgs >> nA_val).astype(np.uint64))
    m = nval_e - nval_a
    ok = (m >= 0) & (m <= nb) & (ncore == (nc - 1 if mode == "ham_n" else 0))
    cfgs, m = cfgs[ok], m[ok]
    full = np.zeros(len(cfgs), dtype=np.int64)
    for i, p in enumerate(a_bits):
        full |= ((cfgs >> i) & 1) << int(p)
    order = np.argsort(full, kind="stable")
    cfgs, m, full = cfgs[order], m[order], full[order]
    sizes = np.array([comb(nb, int(x)) for x in m], dtype=np.int64)
    n_rows = int(sizes.sum())
    nref = len(basis) * (nc if mode == "ham_n" else 1)
    if n_rows != nref or n_rows >= 2 ** 31:
        return None
    slab_off = np.zeros(len(cfgs) + 1, dtype=np.int64)
    slab_off[1:] = np.cumsum(sizes)
    # bath tables
    b_off = np.zeros(nb + 2, dtype=np.int64)
    sect = [_colex(nb, mm) for mm in range(nb + 1)]
    b_off[1:] = np.cumsum([len(s) for s in sect])
    b_cfg = np.concatenate(sect).astype(np.int64)
    rank_of = np.zeros(1 << nb, dtype=np.int64)
    for mm in range(nb + 1):
        rank_of[sect[mm]] = np.arange(len(sect[mm]))
    b_nbr = rank_of[b_cfg[:, None] ^ (1 << np.arange(nb))[None, :]]
    bits = (b_cfg[:, None] >> np.arange(nb)[None, :]) & 1
    b_diag = (bits * b_level[None, :]).sum(axis=1)
    # neighbour slabs
    pos = {int(c): s for s, c in enumerate(cfgs)}
    up = np.full((len(cfgs), nah), -1, dtype=np.int64)
    dn = np.full((len(cfgs), nah), -1, dtype=np.int64)
    for s, c in enumerate(cfgs):
        for q, a in enumerate(act):
            if (c >> a) & 1:
                dn[s, q] = pos.get(int(c & ~(1 << a)), -1)
            else:
                up[s, q] = pos.get(int(c | (1 << a)), -1)
    # permutation: slab row -> reference row
    # fock_core(k) = 2^nc - 1 - 2^(nc-k) has its hole on core orbital nc - k (k = 1..nc,
    # src/ham.f90:419-421); every slab has exactly one hole
    kidx = np.zeros(1 << nc, dtype=np.int64)
    for h in range(nc):
        kidx[((1 << nc) - 1) ^ (1 << h)] = nc - 1 - h
    perm = (_slab_perm_device if on_device else _slab_perm_host)(full, m, sizes, slab_off, b_cfg, b_off, b0, nv,
                                                                 kidx if mode == "ham_n" else None, basis)
    if perm is None:
        return None
    return KronSpec(n=n_rows, nb=nb, b0=int(b0), a_bits=a_bits, n_alo=n_alo,
                    slab_cfg=cfgs.astype(np.uint32), slab_full=full, slab_m=m.astype(np.int32),
                    slab_off=slab_off.astype(np.int32), hyb_a=np.array(act, dtype=np.int32),
                    t_cre=t_cre, t_ann=t_ann, up=up.astype(np.int32), dn=dn.astype(np.int32),
                    b_off=b_off.astype(np.int32), b_cfg=b_cfg.astype(np.uint16), b_nbr=b_nbr.astype(np.uint16),
                    b_diag=b_diag, a_hop=(hi[hop_a] + 1, hv[hop_a]), a_coul=(ci + 1, cv), perm=perm)


def sigma_cre(spec, cfg, m, q):
    """Sign factor of the A side of c+_a c_b on slab cfg (m bath electrons), a = hyb_a[q]."""
    a = int(spec.hyb_a[q])
    lo = (1 << spec.n_alo) - 1
    e = bin(cfg & lo).count("1") + bin(cfg & ((1 << a) - 1)).count("1") + (m - 1 if a >= spec.n_alo else 0)
    return -1.0 if e & 1 else 1.0


def sigma_ann(spec, cfg, m, q):
    """Sign factor of the A side of c+_b c_a on slab cfg (m bath electrons), a = hyb_a[q]."""
    a = int(spec.hyb_a[q])
    lo = (1 << spec.n_alo) - 1
    e = bin(cfg & ((1 << a) - 1)).count("1") + (m if a >= spec.n_alo else 0) + bin(cfg & lo).count("1") - \
        (1 if a < spec.n_alo else 0)
    return -1.0 if e & 1 else 1.0


def apply_np(spec, ha, X):
    """Y = H X in slab order on the host: the restatement of k_lanczos_apply_kron's sums that
    the CPU tests pin against the CSR product.  ha = (row_ptr, col, val) of H_A over the slabs."""
    rp, col, val = ha
    nb = spec.nb
    Y = np.zeros_like(X)
    for s in range(spec.nslab):
        o, e = spec.slab_off[s], spec.slab_off[s + 1]
        mm = int(spec.slab_m[s])
        cfg = int(spec.slab_cfg[s])
        bo = spec.b_off[mm]
        acc = np.zeros((e - o,) + X.shape[1:], dtype=X.dtype)
        for j in range(rp[s], rp[s + 1]):
            t = col[j]
            acc += val[j] * X[spec.slab_off[t]:spec.slab_off[t + 1]]
        d = spec.b_diag[bo:bo + (e - o)]
        acc += d.reshape((-1,) + (1,) * (X.ndim - 1)) * X[o:e]
        for r in range(e - o):
            B = int(spec.b_cfg[bo + r])
            for q in range(spec.nah):
                s2 = spec.up[s, q]
                if s2 >= 0:
                    sa = sigma_cre(spec, cfg, mm, q)
                    for b in range(nb):
                        if (B >> b) & 1 and spec.t_cre[q, b] != 0:
                            sb = -1.0 if bin(B & ((1 << b) - 1)).count("1") & 1 else 1.0
                            acc[r] += sa * sb * spec.t_cre[q, b] * X[spec.slab_off[s2] + spec.b_nbr[bo + r, b]]
                s2 = spec.dn[s, q]
                if s2 >= 0:
                    sa = sigma_ann(spec, cfg, mm, q)
                    for b in range(nb):
                        if not (B >> b) & 1 and spec.t_ann[q, b] != 0:
                            sb = -1.0 if bin(B & ((1 << b) - 1)).count("1") & 1 else 1.0
                            acc[r] += sa * sb * spec.t_ann[q, b] * X[spec.slab_off[s2] + spec.b_nbr[bo + r, b]]
        Y[o:e] = acc
    return Y
