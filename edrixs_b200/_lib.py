"""ctypes binding of libedx.so (the C ABI declared in include/edx.h).

The library is built in-tree by ``edrixs_b200/build.py``.  There is no fallback: if the
shared library is missing or fails to load, every entry point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libedx.so")

EDX_OK = 0
EDX_C128, EDX_C64 = 0, 1
EDX_HAM_I, EDX_HAM_N, EDX_TRANS_I, EDX_TRANS_F = 0, 1, 2, 3
EDX_KRON_AUTO, EDX_KRON_STAGED, EDX_KRON_GATHER = 0, 1, 2  # slab product variants
STATUS = {0: "EDX_OK", 1: "EDX_ERR_INVALID", 2: "EDX_ERR_CUDA", 3: "EDX_ERR_WORKSPACE",
          4: "EDX_ERR_ROW_CAPACITY", 5: "EDX_ERR_OVERFLOW"}

vp = ctypes.c_void_p
i64 = ctypes.c_int64
i32 = ctypes.c_int32
dbl = ctypes.c_double


class EdxError(RuntimeError):
    """A libedx entry point returned a non-zero status."""

    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} -> {STATUS.get(code, code)}: {msg}")
        self.code = code


class BuildDesc(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("fock_left", vp), ("ndim_left", i64), ("fock_right", vp),
                ("ndim_right", i64), ("num_val_orbs", ctypes.c_int), ("num_core_orbs", ctypes.c_int),
                ("search_norb", ctypes.c_int), ("search_nelec", ctypes.c_int), ("nhopp", ctypes.c_int),
                ("hopp_idx", vp), ("hopp_val", vp), ("ncoul", ctypes.c_int), ("coul_idx", vp),
                ("coul_val", vp), ("ham_sign", dbl), ("omega_re", dbl), ("omega_im", dbl)]


class Csr(ctypes.Structure):
    _fields_ = [("nrows", i64), ("ncols", i64), ("nnz", i64), ("row_ptr", vp), ("col", vp), ("val", vp),
                ("val_type", ctypes.c_int)]


class Packed(ctypes.Structure):
    _fields_ = [("nrows", i64), ("nnz", i64), ("row_ptr", vp), ("ent", vp), ("vbits", ctypes.c_int),
                ("nval", ctypes.c_int), ("vals", vp), ("diag", vp), ("vidx", vp)]


class Kron(ctypes.Structure):
    _fields_ = [("nrows", i64), ("nslab", i32), ("nb", i32), ("nah", i32), ("n_alo", i32), ("max_rows", i32),
                ("slab_off", vp), ("slab_m", vp), ("slab_cfg", vp), ("hyb_a", vp), ("t_cre", vp), ("t_ann", vp),
                ("src_ptr", vp), ("src_slab", vp), ("src_kind", vp), ("src_coef", vp), ("b_off", vp), ("b_cfg", vp),
                ("b_nbr", vp), ("b_diag", vp)]


class KrylovOpts(ctypes.Structure):
    _fields_ = [("nproj", ctypes.c_int), ("proj", ctypes.POINTER(Csr)), ("proj_out", ctypes.POINTER(vp)),
                ("nshift", ctypes.c_int), ("shift_col", vp), ("shift_z", vp), ("shift_tol", dbl),
                ("shift_maxit", ctypes.c_int), ("shift_y", vp), ("shift_iters", vp), ("shift_res", vp),
                ("apply_ms", ctypes.POINTER(ctypes.c_double)), ("apply_launches", ctypes.POINTER(ctypes.c_int)),
                ("apply_col_group", ctypes.c_int), ("apply_threads", ctypes.c_int),
                ("apply_blocks_per_sm", ctypes.c_int), ("apply_chunked", ctypes.c_int),
                ("apply_tiles", ctypes.c_int), ("apply_prefetch", ctypes.c_int),
                ("apply_packed", ctypes.POINTER(Packed)), ("apply_kron", ctypes.POINTER(Kron)),
                ("proj_window", ctypes.c_int), ("nacc", ctypes.c_int), ("acc_col", vp), ("acc_coef", vp),
                ("acc_out", ctypes.POINTER(vp)), ("acc_ld", i64), ("v0_ld", i64),
                ("apply_rowslot", ctypes.c_int)]


_SIGS = {
    "edx_last_error": (ctypes.c_char_p, []),
    "edx_abi_version": (ctypes.c_int, []),
    "edx_fock_count": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(i64)]),
    "edx_fock_unrank": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp, i64, vp]),
    "edx_fock_match_full": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp, i64, ctypes.POINTER(ctypes.c_int),
                                           vp, ctypes.c_size_t, vp]),
    "edx_fock_match_full_workspace": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t)]),
    "edx_build_nrows": (i64, [ctypes.POINTER(BuildDesc)]),
    "edx_build_ncols": (i64, [ctypes.POINTER(BuildDesc)]),
    "edx_build_workspace": (ctypes.c_int, [ctypes.POINTER(BuildDesc), ctypes.POINTER(ctypes.c_size_t)]),
    "edx_build_count": (ctypes.c_int, [ctypes.POINTER(BuildDesc), vp, ctypes.POINTER(ctypes.c_int), vp,
                                       ctypes.c_size_t, vp]),
    "edx_build_scan": (ctypes.c_int, [vp, i64, vp, ctypes.POINTER(i64), vp, ctypes.c_size_t, vp]),
    "edx_build_scan_workspace": (ctypes.c_int, [i64, ctypes.POINTER(ctypes.c_size_t)]),
    "edx_build_fill": (ctypes.c_int, [ctypes.POINTER(BuildDesc), ctypes.c_int, vp, vp, vp, vp, vp,
                                      ctypes.c_size_t, vp]),
    "edx_spmm": (ctypes.c_int, [ctypes.POINTER(Csr), ctypes.c_int, ctypes.c_int, vp, i64, vp, i64, dbl, dbl,
                                dbl, dbl, dbl, dbl, ctypes.c_int, vp]),
    "edx_pack_workspace": (ctypes.c_int, [ctypes.POINTER(Csr), ctypes.POINTER(ctypes.c_size_t)]),
    "edx_pack_count": (ctypes.c_int, [ctypes.POINTER(Csr), ctypes.c_int, ctypes.POINTER(i64),
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), vp, ctypes.c_size_t,
                                      vp]),
    "edx_pack_fill": (ctypes.c_int, [ctypes.POINTER(Csr), ctypes.POINTER(Packed), vp, ctypes.c_size_t, vp]),
    "edx_spmm_packed": (ctypes.c_int, [ctypes.POINTER(Packed), ctypes.c_int, vp, i64, vp, i64, dbl, dbl, dbl, dbl,
                                       dbl, dbl, ctypes.c_int, vp]),
    "edx_kron_spmm_workspace": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t)]),
    "edx_kron_spmm": (ctypes.c_int, [ctypes.POINTER(Kron), ctypes.c_int, vp, vp, ctypes.c_int, vp, ctypes.c_size_t,
                                     vp]),
    "edx_permute_rows": (ctypes.c_int, [i64, ctypes.c_int, vp, i64, vp, vp, i64, vp]),
    "edx_proj_combine": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        i64, vp, i64, ctypes.c_int, vp, i64, vp]),
    "edx_gs_workspace": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "edx_gs_dot": (ctypes.c_int, [vp, ctypes.c_int, i64, i64, vp, ctypes.c_int, vp, vp, ctypes.c_size_t, vp]),
    "edx_gs_update": (ctypes.c_int, [vp, ctypes.c_int, i64, i64, vp, ctypes.c_int, vp, vp]),
    "edx_gs_gram": (ctypes.c_int, [vp, i64, ctypes.c_int, vp, vp, ctypes.c_size_t, vp]),
    "edx_gs_rmul": (ctypes.c_int, [vp, i64, ctypes.c_int, vp, vp]),
    "edx_krylov_workspace": (ctypes.c_int, [i64, ctypes.c_int, ctypes.POINTER(KrylovOpts), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_size_t)]),
    "edx_krylov": (ctypes.c_int, [ctypes.POINTER(Csr), ctypes.c_int, vp, ctypes.c_int, vp, vp, vp, vp,
                                  ctypes.POINTER(KrylovOpts), vp, ctypes.c_size_t, vp]),
    "edx_minres_workspace": (ctypes.c_int, [i64, ctypes.POINTER(ctypes.c_size_t)]),
    "edx_minres": (ctypes.c_int, [ctypes.POINTER(Csr), dbl, dbl, dbl, dbl, vp, vp, dbl, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(dbl), vp, ctypes.c_size_t, vp]),
    "edx_cf_spectrum": (ctypes.c_int, [ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp,
                                       vp, vp, ctypes.c_int, ctypes.c_int, vp]),
    "edx_denmat_workspace": (ctypes.c_int, [i64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "edx_denmat": (ctypes.c_int, [vp, i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp,
                                  ctypes.c_size_t, vp]),
    "edx_denmat_static": (ctypes.c_int, [vp, i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp,
                                         vp]),
}

_lib = None


def load():
    """Load libedx.so; raises if it is not there (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libedx.so not found at {LIB_PATH}; build it with "
                          "`python -c 'import __graft_entry__ as g; g.build()'` or edrixs_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols():
    return sorted(_SIGS)


def call(name, *args):
    L = load()
    rc = getattr(L, name)(*args)
    if rc != EDX_OK:
        msg = L.edx_last_error()
        raise EdxError(name, rc, msg.decode() if msg else "")
    return rc
