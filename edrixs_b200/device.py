"""Torch-facing wrappers of the libedx kernels.

Tensors stay on the current CUDA device; every call runs on torch's current stream.
Workspaces are taken from torch's caching allocator, so repeated calls do not hit
cudaMalloc.  Nothing here has a CPU path: without a GPU and libedx.so the calls raise.
"""
import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import BuildDesc, Csr, KrylovOpts, Kron, Packed, call

C128, C64 = _lib.EDX_C128, _lib.EDX_C64
HAM_I, HAM_N, TRANS_I, TRANS_F = _lib.EDX_HAM_I, _lib.EDX_HAM_N, _lib.EDX_TRANS_I, _lib.EDX_TRANS_F
KRON_AUTO, KRON_STAGED, KRON_GATHER = _lib.EDX_KRON_AUTO, _lib.EDX_KRON_STAGED, _lib.EDX_KRON_GATHER


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _work(nbytes):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("edrixs_b200 needs a CUDA device (sm_100a); no CPU path exists")
    _lib.load()


# ------------------------------------------------------------------------------------
# Fock basis
# ------------------------------------------------------------------------------------

@dataclass
class Basis:
    """Ascending Fock states on the device (int64 holding the uint64 bit patterns)."""
    states: torch.Tensor
    norb: int = 0   # >0 when `states` is exactly the full norb/nelec sector
    nelec: int = 0

    @property
    def ndim(self):
        return int(self.states.numel())


def fock_count(norb, nelec):
    n = ctypes.c_int64(0)
    call("edx_fock_count", norb, nelec, ctypes.byref(n))
    return n.value


def fock_unrank(norb, nelec):
    """Full norb/nelec sector in ascending order (replaces get_fock_full_N + sort)."""
    require_cuda()
    n = fock_count(norb, nelec)
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    call("edx_fock_unrank", norb, nelec, _ptr(out), n, _stream())
    return Basis(out, norb, nelec)


def basis_from_states(states):
    """Wrap a sorted state list (e.g. read from fock_*.in); detects the full-sector case."""
    arr = np.asarray(states, dtype=np.uint64)
    if len(arr) > 1 and not np.all(arr[1:] > arr[:-1]):
        # the column search (src/utils.f90:2-40) needs ascending states; unsorted or repeated
        # ones would give wrong matrices without an error
        raise ValueError("basis_from_states: states must be strictly ascending")
    require_cuda()
    t = torch.from_numpy(arr.view(np.int64)).to("cuda")
    b = Basis(t)
    if len(arr) == 0:
        return b
    top = int(arr[-1])
    norb = max(top.bit_length(), 1)
    nelec = bin(int(arr[0])).count("1")
    if norb <= 63:
        ws = ctypes.c_size_t(0)
        call("edx_fock_match_full_workspace", ctypes.byref(ws))
        w = _work(ws.value)
        full = ctypes.c_int(0)
        call("edx_fock_match_full", norb, nelec, _ptr(t), len(arr), ctypes.byref(full), _ptr(w), ws.value,
             _stream())
        if full.value:
            b.norb, b.nelec = norb, nelec
    return b


# ------------------------------------------------------------------------------------
# CSR
# ------------------------------------------------------------------------------------

@dataclass
class CSR:
    row_ptr: torch.Tensor          # int64 [nrows+1]
    col: torch.Tensor              # int32 [nnz]
    val: Optional[torch.Tensor]    # complex128 [nnz] (None for a complex64-only matrix)
    ncols: int
    val64: Optional[torch.Tensor] = None  # complex64 copy (mixed-precision products)

    @property
    def nrows(self):
        return self.row_ptr.numel() - 1

    @property
    def nnz(self):
        return self.col.numel()

    def desc(self, c64=False):
        v = self.val64 if c64 else self.val
        if c64 and v is None:
            raise ValueError("this CSR has no complex64 copy")
        if not c64 and v is None:
            raise ValueError("this CSR holds complex64 values only (use c64=True)")
        return Csr(self.nrows, self.ncols, self.nnz, _ptr(self.row_ptr), _ptr(self.col), _ptr(v),
                   C64 if c64 else C128)

    def nbytes(self, c64=False):
        return self.row_ptr.numel() * 8 + self.nnz * (4 + (8 if c64 else 16))

    def to_c64(self, drop_c128=False, chunk=1 << 28):
        """Add the complex64 copy (converted in chunks, so the peak is the two arrays plus one
        chunk); drop_c128 then releases the complex128 values."""
        if self.val64 is None:
            self.val64 = torch.empty(self.val.numel(), dtype=torch.complex64, device=self.val.device)
            for a in range(0, self.val.numel(), chunk):
                self.val64[a:a + chunk].copy_(self.val[a:a + chunk])
        if drop_c128:
            self.val = None
        return self


def _terms_to_device(terms, nidx):
    if terms is None:
        return None, None, 0
    idx, val = terms
    idx = np.ascontiguousarray(np.asarray(idx, dtype=np.int32).reshape(-1, nidx))
    val = np.ascontiguousarray(np.asarray(val, dtype=np.complex128).reshape(-1))
    return (torch.from_numpy(idx).to("cuda"), torch.from_numpy(val).to("cuda"), len(val))


def build_csr(mode, left: Basis, hopping, coulomb=None, right: Optional[Basis] = None, num_val_orbs=0,
              num_core_orbs=0, ham_sign=1.0, omega=0j, want_c64=False, values=None):
    """Two-pass CSR build of src/ham.f90 (see include/edx.h).  hopping/coulomb are
    (idx 1-based, values) pairs as read from the *.in files.  values: "c128" (default),
    "both" (also a complex64 copy; want_c64=True means the same) or "c64" (complex64 only,
    for matrices too large to hold in complex128)."""
    values = values or ("both" if want_c64 else "c128")
    if values not in ("c128", "c64", "both"):
        raise ValueError("build_csr: values must be c128, c64 or both")
    require_cuda()
    hi, hv, nh = _terms_to_device(hopping, 2)
    ci, cv, ncl = _terms_to_device(coulomb, 4)
    search = right if mode in (TRANS_I, TRANS_F) else left
    d = BuildDesc(mode, _ptr(left.states), left.ndim, _ptr(right.states) if right is not None else None,
                  right.ndim if right is not None else 0, num_val_orbs, num_core_orbs, search.norb, search.nelec,
                  nh, _ptr(hi), _ptr(hv), ncl, _ptr(ci), _ptr(cv), float(ham_sign), float(np.real(omega)),
                  float(np.imag(omega)))
    L = _lib.load()
    nrows = L.edx_build_nrows(ctypes.byref(d))
    ncols = L.edx_build_ncols(ctypes.byref(d))
    ws = ctypes.c_size_t(0)
    call("edx_build_workspace", ctypes.byref(d), ctypes.byref(ws))
    sws = ctypes.c_size_t(0)
    call("edx_build_scan_workspace", nrows, ctypes.byref(sws))
    w = _work(max(ws.value, sws.value))
    row_nnz = torch.empty(nrows, dtype=torch.int32, device="cuda")
    cap = ctypes.c_int(0)
    st = _stream()
    call("edx_build_count", ctypes.byref(d), _ptr(row_nnz), ctypes.byref(cap), _ptr(w), ws.value, st)
    row_ptr = torch.empty(nrows + 1, dtype=torch.int64, device="cuda")
    nnz = ctypes.c_int64(0)
    call("edx_build_scan", _ptr(row_nnz), nrows, _ptr(row_ptr), ctypes.byref(nnz), _ptr(w), sws.value, st)
    del row_nnz
    col = torch.empty(max(nnz.value, 1), dtype=torch.int32, device="cuda")[:nnz.value]
    val = torch.empty(max(nnz.value, 1), dtype=torch.complex128, device="cuda")[:nnz.value] \
        if values != "c64" else None
    val64 = torch.empty(max(nnz.value, 1), dtype=torch.complex64, device="cuda")[:nnz.value] \
        if values != "c128" else None
    if nnz.value > 0:
        call("edx_build_fill", ctypes.byref(d), cap.value, _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(val64),
             _ptr(w), ws.value, st)
    # the term tensors may be released now: the caching allocator only reuses their memory
    # for work queued later on this stream, after the fill kernel
    return CSR(row_ptr, col, val, ncols, val64)


# ------------------------------------------------------------------------------------
# packed form (edx_pack_*)
# ------------------------------------------------------------------------------------

PACK_VALUES_MAX = 2048


@dataclass
class PackedMatrix:
    """Device arrays of an edx_packed matrix (see include/edx.h); keeps them alive."""
    row_ptr: torch.Tensor   # int64 [n+1], off-diagonal entries
    ent: torch.Tensor       # int32 [nnz]: uint32 words column << vbits | value index (narrow),
                            # or the column (wide, vbits == 0)
    vals: torch.Tensor      # complex128 [nval]
    diag: torch.Tensor      # complex128 [n]
    vbits: int
    vidx: Optional[torch.Tensor] = None  # int16 [nnz] holding uint16 value indices (wide form)

    @property
    def nrows(self):
        return self.row_ptr.numel() - 1

    ncols = nrows

    @property
    def nnz(self):
        return self.ent.numel()

    @property
    def wide(self):
        return self.vbits == 0

    def desc(self):
        return Packed(self.nrows, self.ent.numel(), _ptr(self.row_ptr), _ptr(self.ent), self.vbits,
                      self.vals.numel(), _ptr(self.vals), _ptr(self.diag),
                      _ptr(self.vidx) if self.vidx is not None else None)

    def shape_desc(self):
        """A CSR descriptor with this matrix's shape and no entries, for calls whose product
        runs on the packed form (edx_krylov with apply_packed)."""
        return Csr(self.nrows, self.nrows, 0, _ptr(self.row_ptr), None, None, C128)

    def nbytes(self):
        ts = [self.row_ptr, self.ent, self.vals, self.diag] + ([self.vidx] if self.vidx is not None else [])
        return sum(t.numel() * t.element_size() for t in ts)

    def unpack(self):
        """(row_ptr, col, val) of the off-diagonal entries, for checks."""
        w = self.ent.to(torch.int64) & 0xFFFFFFFF
        if self.wide:
            return self.row_ptr, w, self.vals[self.vidx.to(torch.int64) & 0xFFFF]
        return self.row_ptr, (w >> self.vbits), self.vals[w & ((1 << self.vbits) - 1)]


PACK_FORMS = {"auto": 0, "narrow": 1, "wide": 2}


def pack(A: CSR, form="auto"):
    """Packed form of the square complex128 matrix A, or None when A has more distinct
    off-diagonal values than the form can index.  form: "auto" (the 32-bit word when the
    column leaves room for the value index, else the wide form), "narrow" or "wide"."""
    require_cuda()
    d = A.desc()
    ws = ctypes.c_size_t(0)
    call("edx_pack_workspace", ctypes.byref(d), ctypes.byref(ws))
    w = _work(ws.value)
    nnz, nval, vbits = ctypes.c_int64(0), ctypes.c_int(0), ctypes.c_int(0)
    st = _stream()
    try:
        call("edx_pack_count", ctypes.byref(d), PACK_FORMS[form], ctypes.byref(nnz), ctypes.byref(nval),
             ctypes.byref(vbits), _ptr(w), ws.value, st)
    except _lib.EdxError as e:
        if e.code == 5:  # EDX_ERR_OVERFLOW: too many distinct values
            return None
        raise
    n = A.nrows
    m = nnz.value
    P = PackedMatrix(torch.empty(n + 1, dtype=torch.int64, device="cuda"),
                     torch.empty(max(m, 1), dtype=torch.int32, device="cuda")[:m],
                     torch.empty(max(nval.value, 1), dtype=torch.complex128, device="cuda")[:nval.value],
                     torch.empty(n, dtype=torch.complex128, device="cuda"), vbits.value,
                     torch.empty(max(m, 1), dtype=torch.int16, device="cuda")[:m] if vbits.value == 0 else None)
    t = P.desc()
    call("edx_pack_fill", ctypes.byref(d), ctypes.byref(t), _ptr(w), ws.value, st)
    return P


# ------------------------------------------------------------------------------------
# products and solvers
# ------------------------------------------------------------------------------------

# ------------------------------------------------------------------------------------
# slab form (edx_kron_*)
# ------------------------------------------------------------------------------------

KRON_SRC_HA, KRON_SRC_OWN, KRON_SRC_CRE, KRON_SRC_ANN = 0, 1, 2, 3


@dataclass
class KronMatrix:
    """Device arrays of the slab form of a Hamiltonian (edrixs_b200/kron.py, include/edx.h
    edx_kron); its rows and columns are in slab order.  perm[i] is the reference row of slab
    row i, inv its inverse."""
    spec: object
    nrows: int
    max_rows: int
    t: dict
    perm: torch.Tensor
    inv: torch.Tensor

    def desc(self):
        t = self.t
        return Kron(self.nrows, self.spec.nslab, self.spec.nb, self.spec.nah, self.spec.n_alo, self.max_rows,
                    _ptr(t["slab_off"]), _ptr(t["slab_m"]), _ptr(t["slab_cfg"]), _ptr(t["hyb_a"]), _ptr(t["t_cre"]),
                    _ptr(t["t_ann"]), _ptr(t["src_ptr"]), _ptr(t["src_slab"]), _ptr(t["src_kind"]),
                    _ptr(t["src_coef"]), _ptr(t["b_off"]), _ptr(t["b_cfg"]), _ptr(t["b_nbr"]), _ptr(t["b_diag"]))

    def shape_desc(self):
        """A CSR descriptor with this matrix's shape and no entries, for edx_krylov with
        apply_kron (the product runs on the slab form)."""
        return Csr(self.nrows, self.nrows, 0, _ptr(self.t["slab_off"]), None, None, C128)

    def nbytes(self):
        return sum(x.numel() * x.element_size() for x in self.t.values()) + 16 * self.nrows

    @property
    def nnz(self):
        return 0

    def to_slab(self, X):
        """Rows of X (reference order) in slab order."""
        return permute_rows(X, self.perm)

    def from_slab(self, X):
        """Rows of X (slab order) in reference order."""
        return permute_rows(X, self.inv)


def kron_form(mode, basis: Basis, hopping, coulomb=None, num_val_orbs=0, num_core_orbs=0):
    """The slab form of the Hamiltonian that build_csr(mode, basis, hopping, coulomb, ...)
    builds (HAM_I, or HAM_N with ham_sign = +1), or None when the terms have no impurity x bath
    structure.  H_A is built by the same bit-exact build on the A configurations."""
    from . import kron
    if mode not in (HAM_I, HAM_N):
        return None
    spec = kron.kron_spec(hopping, coulomb, basis.states, "ham_i" if mode == HAM_I else "ham_n",
                          num_val_orbs=num_val_orbs, num_core_orbs=num_core_orbs)
    if spec is None:
        return None
    # rows are A configurations as full-state bit patterns (valence and core bits in place)
    HA = build_csr(HAM_I, basis_from_states(spec.slab_full.astype(np.uint64)), spec.a_hop,
                   spec.a_coul if len(spec.a_coul[1]) else None, num_val_orbs=num_val_orbs + num_core_orbs)
    rp, col, val = HA.row_ptr.cpu().numpy(), HA.col.cpu().numpy(), HA.val.cpu().numpy()
    # per-slab source list: the slab itself (H_A's diagonal + bath levels), H_A's other
    # columns, then the slabs one bath electron away
    has_cre = np.any(spec.t_cre != 0, axis=1)
    has_ann = np.any(spec.t_ann != 0, axis=1)
    ptr, sl, kind, coef = [0], [], [], []
    for s in range(spec.nslab):
        j0, j1 = rp[s], rp[s + 1]
        cs, vs = col[j0:j1], val[j0:j1]
        d = vs[cs == s]
        sl.append(s)
        kind.append(KRON_SRC_OWN)
        coef.append(d[0] if len(d) else 0j)
        off = cs != s
        sl.extend(cs[off].tolist())
        kind.extend([KRON_SRC_HA] * int(off.sum()))
        coef.extend(vs[off].tolist())
        for q in range(spec.nah):
            u, dn = spec.up[s, q], spec.dn[s, q]
            if u >= 0 and has_cre[q]:
                sl.append(int(u))
                kind.append(KRON_SRC_CRE | (q << 4))
                coef.append(0j)
            if dn >= 0 and has_ann[q]:
                sl.append(int(dn))
                kind.append(KRON_SRC_ANN | (q << 4))
                coef.append(0j)
        ptr.append(len(sl))
    dev = dict(device="cuda")

    def i32(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64).astype(np.int32), **dev)

    def c128(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.complex128).reshape(-1), **dev)

    def u16(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.uint16).reshape(-1).view(np.int16), **dev)

    t = dict(slab_off=i32(spec.slab_off), slab_m=i32(spec.slab_m), slab_cfg=i32(spec.slab_cfg),
             hyb_a=i32(spec.hyb_a if spec.nah else [0]), t_cre=c128(spec.t_cre if spec.nah else [0j]),
             t_ann=c128(spec.t_ann if spec.nah else [0j]),
             src_ptr=torch.as_tensor(np.asarray(ptr, dtype=np.int64), **dev), src_slab=i32(sl), src_kind=i32(kind),
             src_coef=c128(coef), b_off=i32(spec.b_off), b_cfg=u16(spec.b_cfg), b_nbr=u16(spec.b_nbr),
             b_diag=c128(spec.b_diag))
    perm = torch.as_tensor(spec.perm, dtype=torch.int64, **dev)
    inv = torch.empty_like(perm)
    inv[perm] = torch.arange(spec.n, dtype=torch.int64, **dev)
    return KronMatrix(spec, spec.n, spec.max_rows, t, perm, inv)


def relabel_columns(D: CSR, idx):
    """D with column j renamed idx[j] (row pointers and values shared): an operator whose
    columns were in the reference's row order of a matrix, re-expressed on that matrix's slab
    order (idx = KronMatrix.inv).  Rows keep their entry order, so each row's sum is taken in
    the same order as on D."""
    col = idx.index_select(0, D.col.to(torch.int64)).to(torch.int32)
    return CSR(D.row_ptr, col, D.val, D.ncols, D.val64)


def permute_rows(X, idx):
    """Y[i] = X[idx[i]] (rows of a complex128 block), by libedx's edx_permute_rows."""
    Xm = X.reshape(X.shape[0], -1)
    if Xm.stride(1) != 1 and Xm.shape[1] > 1:
        Xm = Xm.contiguous()
    n, k = idx.numel(), Xm.shape[1]
    Y = torch.empty((n, k), dtype=torch.complex128, device=X.device)
    call("edx_permute_rows", n, k, _ptr(Xm), Xm.stride(0), _ptr(idx), _ptr(Y), k, _stream())
    return Y.reshape(-1) if X.dim() == 1 else Y


def proj_combine(projs, y, k, nw, m):
    """Final-state start vectors from stored projections (edx_proj_combine): returns the
    row-major (nrows, len(projs) * k * nw) block with column (p * k + c) * nw + w equal to
    sum_{i < m} y[c * nw + w, i] * projs[p][c, i, :].  projs: (k, steps, nrows) complex128
    blocks with rows contiguous, such as krylov's stored projections (views of (k, maxn,
    nrows) buffers); y: (k * nw, ldy) complex128 with ldy >= m."""
    np_ = len(projs)
    kk, steps, nrows = projs[0].shape
    if kk != k or y.shape[0] != k * nw or y.stride(1) != 1 or y.dtype != torch.complex128 or m > steps:
        raise ValueError("proj_combine: shapes or layout do not match")
    cstride = projs[0].stride(0)
    for P in projs:
        if (tuple(P.shape) != (k, steps, nrows) or P.stride(2) != 1 or P.stride(1) != nrows or P.stride(0) != cstride
                or cstride % nrows or P.dtype != torch.complex128):
            raise ValueError("proj_combine: projections must be (k, steps, nrows) complex128 blocks of contiguous "
                             "rows with one column stride")
    out = torch.empty((nrows, np_ * k * nw), dtype=torch.complex128, device=y.device)
    ptrs = (ctypes.c_void_p * np_)(*[P.data_ptr() for P in projs])
    call("edx_proj_combine", np_, ptrs, k, cstride // nrows, int(m), nrows, _ptr(y), y.stride(0), nw, _ptr(out),
         out.stride(0), _stream())
    return out


def spmm(A, X, Y=None, alpha=1.0, sigma=0.0, beta=0.0, c64=False, col_group=0):
    """Y = alpha*(A X) + sigma*X + beta*Y; X is (ncols,) or (ncols, k) row-major.  A is a CSR
    or a PackedMatrix (edx_spmm_packed)."""
    squeeze = X.dim() == 1
    Xm = X.reshape(X.shape[0], -1)
    k = Xm.shape[1]
    if Y is None:
        Y = torch.zeros((A.nrows, k), dtype=X.dtype, device=X.device)
        beta = 0.0
    Ym = Y.reshape(Y.shape[0], -1)
    vec_type = C64 if X.dtype == torch.complex64 else C128
    # rows must be contiguous; a single column's stride is irrelevant (torch leaves a (n, 1)
    # slice of a column-major block with column stride n, and calls it contiguous)
    if k > 1 and Xm.stride(1) != 1:
        Xm = Xm.contiguous()
    if k > 1 and Ym.stride(1) != 1:
        raise ValueError("spmm: Y must be row-major (n, k)")
    al, sg, be = complex(alpha), complex(sigma), complex(beta)
    if isinstance(A, KronMatrix):
        if vec_type != C128 or c64 or al != 1 or sg != 0 or be != 0 or Xm.stride(0) != k or Ym.stride(0) != k:
            raise ValueError("spmm: the slab form computes Y = H X on contiguous complex128 blocks only")
        ws = ctypes.c_size_t(0)
        call("edx_kron_spmm_workspace", ctypes.byref(ws))
        w = _work(ws.value)
        call("edx_kron_spmm", ctypes.byref(A.desc()), k, _ptr(Xm), _ptr(Ym), col_group, _ptr(w), ws.value,
             _stream())
    elif isinstance(A, PackedMatrix):
        if vec_type != C128 or c64:
            raise ValueError("spmm: a packed matrix takes complex128 vectors")
        call("edx_spmm_packed", ctypes.byref(A.desc()), k, _ptr(Xm), Xm.stride(0), _ptr(Ym), Ym.stride(0),
             al.real, al.imag, sg.real, sg.imag, be.real, be.imag, col_group, _stream())
    else:
        call("edx_spmm", ctypes.byref(A.desc(c64)), k, vec_type, _ptr(Xm), Xm.stride(0), _ptr(Ym), Ym.stride(0),
             al.real, al.imag, sg.real, sg.imag, be.real, be.imag, col_group, _stream())
    return Y.reshape(-1) if squeeze else Y


@dataclass
class KrylovResult:
    alpha: torch.Tensor   # (k, maxn) float64 (device)
    beta: torch.Tensor    # (k, maxn)
    norm: torch.Tensor    # (k,)
    neff: torch.Tensor    # (k,) int32
    proj: list            # per projector: (k, steps + 1 (<= maxn), nrows_p) complex128
    shift_y: Optional[torch.Tensor] = None      # (nshift, maxn) complex128
    shift_iters: Optional[torch.Tensor] = None
    shift_res: Optional[torch.Tensor] = None


def krylov(A, V0, maxn, c64=False, proj=(), shifts=None, shift_tol=1e-10, shift_maxit=None, timing=False,
           apply=None, accumulate=None):
    """k independent Lanczos recurrences (build_krylov_mp) from the columns of V0 (n, k).
    proj: CSR operators applied to every Lanczos vector.  shifts: (col_index int array,
    complex z array) -> per-shift MINRES coefficients in the Lanczos basis.  A may be a
    PackedMatrix: the product then runs on it and no CSR is needed.
    accumulate: dict(window=B, col=(nacc,) ints, coef=(nacc, maxn) complex128 device tensor,
    out=[one (nrows_p, nacc) row-major view per projector]) -> instead of storing every
    projected vector, out[p][:, s] += sum_i coef[s, i] * (proj[p] v_i)[:, col[s]], keeping
    only the last B projected vectors."""
    if isinstance(A, PackedMatrix):
        apply = dict(apply or {}, packed=A)
    if isinstance(A, KronMatrix):
        apply = dict(apply or {}, kron=A)
    kcols = V0.reshape(V0.shape[0], -1).shape[1]
    if apply and apply.get("packed") is not None and "rowslot" not in apply and kcols <= 16 \
            and "col_group" not in apply:
        # a few columns on the packed form: one row per lane group, the measured best shape
        th = int(apply.get("threads", 256))
        apply = dict({"threads": th, "blocks_per_sm": 4 if th == 256 else 1}, **apply, rowslot=1)
    V0 = V0.reshape(V0.shape[0], -1)
    if (V0.shape[1] > 1 and V0.stride(1) != 1) or V0.stride(0) < V0.shape[1]:
        V0 = V0.contiguous()
    n, k = V0.shape
    dev = V0.device
    alpha = torch.zeros((k, maxn), dtype=torch.float64, device=dev)
    beta = torch.zeros((k, maxn), dtype=torch.float64, device=dev)
    norm = torch.zeros(k, dtype=torch.float64, device=dev)
    neff = torch.zeros(k, dtype=torch.int32, device=dev)
    opts = KrylovOpts()
    opts.v0_ld = V0.stride(0)  # the start vectors may be columns of a wider row-major block
    keep = []
    outs = []
    if proj:
        depth = int(accumulate["window"]) if accumulate else maxn
        descs = (Csr * len(proj))(*[P.desc() for P in proj])
        # every slot that is returned gets written: no clearing pass over what can be tens of GB
        outs = [torch.empty((k, depth, P.nrows), dtype=torch.complex128, device=dev) for P in proj]
        ptrs = (ctypes.c_void_p * len(proj))(*[o.data_ptr() for o in outs])
        opts.nproj = len(proj)
        opts.proj = descs
        opts.proj_out = ptrs
        keep += [descs, ptrs]
        if accumulate:
            acc_col = torch.as_tensor(np.asarray(accumulate["col"], dtype=np.int32), device=dev)
            coef = accumulate["coef"]
            aouts = accumulate["out"]
            nacc = acc_col.numel()
            if coef.dtype != torch.complex128 or tuple(coef.shape) != (nacc, maxn) or not coef.is_contiguous():
                raise ValueError("krylov: accumulate coef must be a contiguous (nacc, maxn) complex128 tensor")
            if len(aouts) != len(proj):
                raise ValueError("krylov: one accumulator block per projector")
            ld = aouts[0].stride(0)
            for P, o in zip(proj, aouts):
                if o.dtype != torch.complex128 or tuple(o.shape) != (P.nrows, nacc) or o.stride(1) != 1 \
                        or o.stride(0) != ld:
                    raise ValueError("krylov: accumulator blocks must be (nrows_p, nacc) row-major views, one ld")
            aptrs = (ctypes.c_void_p * len(proj))(*[o.data_ptr() for o in aouts])
            opts.proj_window = depth
            opts.nacc = nacc
            opts.acc_col = _ptr(acc_col)
            opts.acc_coef = _ptr(coef)
            opts.acc_out = aptrs
            opts.acc_ld = ld
            keep += [acc_col, aptrs]
    sy = si = sr = None
    if shifts is not None:
        scol, sz = shifts
        scol_t = torch.as_tensor(np.asarray(scol, dtype=np.int32), device=dev)
        sz_t = torch.as_tensor(np.asarray(sz, dtype=np.complex128), device=dev)
        ns = scol_t.numel()
        sy = torch.zeros((ns, maxn), dtype=torch.complex128, device=dev)
        si = torch.zeros(ns, dtype=torch.int32, device=dev)
        sr = torch.zeros(ns, dtype=torch.float64, device=dev)
        opts.nshift = ns
        opts.shift_col = _ptr(scol_t)
        opts.shift_z = _ptr(sz_t)
        opts.shift_tol = float(shift_tol)
        opts.shift_maxit = int(shift_maxit if shift_maxit is not None else maxn)
        opts.shift_y = _ptr(sy)
        opts.shift_iters = _ptr(si)
        opts.shift_res = _ptr(sr)
        keep += [scol_t, sz_t]
    if apply:
        opts.apply_col_group = int(apply.get("col_group", 0))
        opts.apply_threads = int(apply.get("threads", 0))
        opts.apply_blocks_per_sm = int(apply.get("blocks_per_sm", 0))
        opts.apply_chunked = int(apply.get("chunked", 0))
        opts.apply_tiles = int(apply.get("tiles", 0))
        opts.apply_prefetch = int(apply.get("prefetch", 0))
        opts.apply_rowslot = int(apply.get("rowslot", 0))
        if apply.get("packed") is not None:
            pdesc = apply["packed"].desc()
            opts.apply_packed = ctypes.pointer(pdesc)
            keep += [pdesc]
        if apply.get("kron") is not None:
            kdesc = apply["kron"].desc()
            opts.apply_kron = ctypes.pointer(kdesc)
            keep += [kdesc]
    ms = ctypes.c_double(0.0)
    nl = ctypes.c_int(0)
    if timing:
        opts.apply_ms = ctypes.pointer(ms)
    opts.apply_launches = ctypes.pointer(nl)
    ws = ctypes.c_size_t(0)
    call("edx_krylov_workspace", n, k, ctypes.byref(opts), maxn, ctypes.byref(ws))
    w = _work(ws.value)
    adesc = A.shape_desc() if isinstance(A, (PackedMatrix, KronMatrix)) else A.desc(c64)
    call("edx_krylov", ctypes.byref(adesc), k, _ptr(V0), maxn, _ptr(alpha), _ptr(beta), _ptr(norm),
         _ptr(neff), ctypes.byref(opts), _ptr(w), ws.value, _stream())
    # projected vectors exist for v_0 .. v_L after L iterations
    written = min(nl.value + 1, maxn)
    res = KrylovResult(alpha, beta, norm, neff, [] if accumulate else [o[:, :written, :] for o in outs], sy, si, sr)
    res.apply_ms = ms.value if timing else None
    res.apply_launches = nl.value
    return res


def minres(A: CSR, b, tol, maxit, alpha=1.0, sigma=0.0, c64=False):
    """pminres_csr on op(A) = alpha*A + sigma*I; returns (x, iterations, |res| estimate)."""
    n = A.nrows
    x = torch.zeros(n, dtype=torch.complex128, device=b.device)
    ws = ctypes.c_size_t(0)
    call("edx_minres_workspace", n, ctypes.byref(ws))
    w = _work(ws.value)
    it = ctypes.c_int(0)
    res = ctypes.c_double(0)
    al, sg = complex(alpha), complex(sigma)
    b = b.contiguous()
    call("edx_minres", ctypes.byref(A.desc(c64)), al.real, al.imag, sg.real, sg.imag, _ptr(b), _ptr(x),
         float(tol), int(maxit), ctypes.byref(it), ctypes.byref(res), _ptr(w), ws.value, _stream())
    return x, it.value, res.value


def gs_dot(V, m, W):
    """C = V[:m]^H W for V (>= m, n) row-major basis vectors and W (n, k) row-major, k <= 8."""
    n, k = W.shape
    assert V.stride(1) == 1 and W.is_contiguous() and V.shape[1] == n
    C = torch.empty((m, k), dtype=torch.complex128, device=W.device)
    ws = ctypes.c_size_t(0)
    call("edx_gs_workspace", m, k, ctypes.byref(ws))
    w = _work(ws.value)
    call("edx_gs_dot", _ptr(V), m, n, V.stride(0), _ptr(W), k, _ptr(C), _ptr(w), ws.value, _stream())
    return C


def gs_gram(W):
    """G = W^H W (k x k) for a row-major (n, k) block, k <= 8."""
    n, k = W.shape
    assert W.is_contiguous()
    G = torch.empty((k, k), dtype=torch.complex128, device=W.device)
    ws = ctypes.c_size_t(0)
    call("edx_gs_workspace", k, k, ctypes.byref(ws))
    w = _work(ws.value)
    call("edx_gs_gram", _ptr(W), n, k, _ptr(G), _ptr(w), ws.value, _stream())
    return G


def gs_rmul(W, M):
    """W = W M in place for a row-major (n, k) block and a (k, k) matrix."""
    n, k = W.shape
    assert W.is_contiguous()
    Mc = torch.as_tensor(M, dtype=torch.complex128).to(W.device).contiguous()
    call("edx_gs_rmul", _ptr(W), n, k, _ptr(Mc), _stream())
    return W


def gs_update(V, m, W, C):
    """W -= V[:m]^T C in place."""
    n, k = W.shape
    assert V.stride(1) == 1 and W.is_contiguous() and V.shape[1] == n
    Cc = C.contiguous()
    call("edx_gs_update", _ptr(V), m, n, V.stride(0), _ptr(W), k, _ptr(Cc), _stream())
    return W


def cf_spectrum(neff, alpha, beta, e0, norm, weight, omega, gamma, per_set=False):
    """Continued fraction of get_spectra_from_poles on the device.
    alpha/beta: (nset, ld) float64; returns (ngrid,) or (nset, ngrid)."""
    nset, ld = alpha.shape
    dev = alpha.device
    f64 = dict(dtype=torch.float64, device=dev)
    omega = torch.as_tensor(omega, **f64).contiguous()
    if not torch.is_tensor(gamma):  # a numpy broadcast view is read-only: copy it first
        gamma = np.array(gamma, dtype=np.float64)
    gamma = torch.broadcast_to(torch.as_tensor(gamma, **f64), omega.shape).contiguous()
    out = torch.zeros((nset, omega.numel()) if per_set else (omega.numel(),), **f64)
    # every argument tensor is bound to a name: a temporary freed before the launch could
    # hand its memory to the next argument
    neff_t = neff.to(torch.int32).contiguous()
    alpha_t, beta_t = alpha.contiguous(), beta.contiguous()
    e0_t = torch.as_tensor(np.asarray(e0, dtype=np.float64), **f64).contiguous()
    norm_t = torch.as_tensor(np.asarray(norm, dtype=np.float64) if not torch.is_tensor(norm) else norm,
                             **f64).contiguous()
    w_t = torch.as_tensor(np.asarray(weight, dtype=np.float64), **f64).contiguous()
    call("edx_cf_spectrum", nset, _ptr(neff_t), _ptr(alpha_t), _ptr(beta_t), ld, _ptr(e0_t), _ptr(norm_t),
         _ptr(w_t), omega.numel(), _ptr(omega), _ptr(gamma), _ptr(out), 1 if per_set else 0, 0, _stream())
    return out


def denmat(basis: Basis, nv, vecs):
    """<c+_i c_j> per eigenvector (ed_driver.f90:194-248): vecs (n, nvec) -> (nvec, nv, nv)."""
    vecs = vecs.reshape(vecs.shape[0], -1).contiguous()
    n, nvec = vecs.shape
    out = torch.zeros((nvec, nv, nv), dtype=torch.complex128, device=vecs.device)
    ws = ctypes.c_size_t(0)
    call("edx_denmat_workspace", n, nv, nvec, ctypes.byref(ws))
    w = _work(ws.value)
    call("edx_denmat", _ptr(basis.states), n, basis.norb, basis.nelec, nv, nvec, _ptr(vecs), _ptr(out), _ptr(w),
         ws.value, _stream())
    return out
