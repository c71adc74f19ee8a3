"""CPU tests: drop-in file formats, the C ABI surface, and the seeded workload generator."""
import os
import re
import struct

import numpy as np
import pytest

from edrixs_b200 import io as edxio
from edrixs_b200 import siam

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# ---- config.in namelist (src/io.f90:2-67) -------------------------------------------

def test_config_partial_namelist(golden_dir):
    cfg = edxio.read_config(os.path.join(golden_dir, "known_answer", "config.in"))
    assert cfg["ed_solver"] == 0 and cfg["num_val_orbs"] == 20 and cfg["neval"] == 45
    assert cfg["idump"] is True and cfg["eigval_tol"] == 1e-10
    # keys absent from the file keep the Fortran defaults (io.f90:17-32)
    assert cfg["linsys_max"] == 500 and cfg["nkryl"] == 500 and cfg["gamma_in"] == 0.1


def test_config_variants(tmp_path):
    p = tmp_path / "config.in"
    p.write_text("&CONTROL\n ed_solver = 2, neval=3 ! comment\n linsys_tol=1d-12\n idump=T\n"
                 " omega_in = -1.5E+00\n/\n")
    cfg = edxio.read_config(str(p))
    assert cfg["ed_solver"] == 2 and cfg["neval"] == 3 and cfg["linsys_tol"] == 1e-12
    assert cfg["idump"] is True and cfg["omega_in"] == -1.5
    p.write_text("&control\nbogus_key=1\n&end\n")
    with pytest.raises(edxio.EdxInputError):
        edxio.read_config(str(p))


def test_missing_file_raises(tmp_path):
    with pytest.raises(edxio.EdxInputError, match="hopping_i.in doesn't exist"):
        edxio.read_hopping(str(tmp_path / "hopping_i.in"))


@pytest.mark.parametrize("text,msg", [
    ("abc\n1 1 0.5 0\n", "count"), ("-2\n1 1 0.5 0\n", "negative count"),
    ("2\n1 1 0.5 0\n", "short"), ("1\nx 1 0.5 0\n", "malformed term"),
    ("1\n1.5 1 0.5 0\n", "malformed term"), ("1\n1 1 zz 0\n", "malformed term"),
    ("1\n0 1 0.5 0\n", "1..64"),
])
def test_malformed_term_files_raise_input_errors(tmp_path, text, msg):
    """A malformed hopping / Coulomb / transition file fails with EdxInputError naming the
    file, where the reference STOPs (src/io.f90:86-89)."""
    p = tmp_path / "hopping_i.in"
    p.write_text(text)
    with pytest.raises(edxio.EdxInputError, match=msg):
        edxio.read_hopping(str(p))


@pytest.mark.parametrize("text,msg", [
    ("3\n1\n2\n", "short"), ("2\n3\n1\n", "ascending"), ("2\n1\n1\n", "ascending"),
    ("2\n1\nx\n", "malformed state"), ("x\n1\n", "count"),
])
def test_malformed_fock_files_raise_input_errors(tmp_path, text, msg):
    """The reference's writer sorts the basis (edrixs/fock_basis.py:444) and its column search
    relies on it (src/utils.f90:2-40), so an unsorted or repeated list is rejected."""
    p = tmp_path / "fock_i.in"
    p.write_text(text)
    with pytest.raises(edxio.EdxInputError, match=msg):
        edxio.read_fock(str(p))


def test_reference_caller_files_parse(golden_dir):
    d = os.path.join(golden_dir, "siam_callers", "rixs_2")
    cfg = edxio.read_config(os.path.join(d, "config.in"))
    assert cfg["num_core_orbs"] == 6 and cfg["linsys_tol"] == 1e-10 and cfg["nkryl"] == 50
    fi = edxio.read_fock(os.path.join(d, "fock_i.in"))
    assert len(fi) == 120 and np.all(np.diff(fi.astype(np.int64)) > 0)
    idx, val = edxio.read_hopping(os.path.join(d, "transop_rixs_f.in"))
    assert idx.shape[1] == 2 and idx.min() >= 1
    idx, val = edxio.read_coulomb(os.path.join(d, "coulomb_n.in"))
    assert idx.shape[1] == 4 and len(val) > 340


def test_writers_byte_identical_to_reference_callers(golden_dir, tmp_path):
    """config.in and fock_i.in written by this package == the reference's own writers."""
    d = os.path.join(golden_dir, "siam_callers", "rixs_2")
    cfg = edxio.read_config(os.path.join(d, "config.in"))
    edxio.write_config(str(tmp_path), num_val_orbs=cfg["num_val_orbs"], num_core_orbs=6,
                       omega_in=float(open(os.path.join(d, "config.in")).read().split("omega_in=")[1].split()[0]),
                       gamma_in=cfg["gamma_in"], num_gs=1, nkryl=50, linsys_max=500, linsys_tol=1e-10)
    assert open(tmp_path / "config.in").read() == open(os.path.join(d, "config.in")).read()
    edxio.write_fock(str(tmp_path / "fock_i.in"), siam.fock_states(10, 3))
    assert open(tmp_path / "fock_i.in").read() == open(os.path.join(d, "fock_i.in")).read()


def test_emat_writer_matches_reference_text(golden_dir, tmp_path):
    d = os.path.join(golden_dir, "siam_callers", "rixs_2")
    idx, val = edxio.read_hopping(os.path.join(d, "hopping_n.in"))
    n = idx.max()
    e = np.zeros((16, 16), dtype=complex)
    e[idx[:, 0] - 1, idx[:, 1] - 1] = val
    edxio.write_emat(e, str(tmp_path / "h.in"))
    ours = open(tmp_path / "h.in").read().splitlines()
    ref = open(os.path.join(d, "hopping_n.in")).read().splitlines()
    assert len(ours) == len(ref) and ours[0] == ref[0]
    for a, b in zip(ours[1:], ref[1:]):
        fa, fb = a.split(), b.split()
        assert fa[:2] == fb[:2]
        assert abs(float(fa[2]) - float(fb[2])) < 1e-14 and abs(float(fa[3]) - float(fb[3])) < 1e-14
    assert n <= 16


def test_empty_operator_placeholder(tmp_path):
    edxio.write_emat(np.zeros((4, 4)), str(tmp_path / "e.in"))
    idx, val = edxio.read_hopping(str(tmp_path / "e.in"))
    assert idx.tolist() == [[1, 1]] and val.tolist() == [0j]


def test_eigvec_roundtrip_and_fortran_layout(tmp_path):
    v = (np.arange(7) + 1j * np.arange(7)[::-1]).astype(np.complex128)
    p = str(tmp_path / "eigvec.1")
    edxio.write_eigvec(p, -3.25, v)
    raw = open(p, "rb").read()
    assert struct.unpack_from("<i", raw, 0)[0] == 8 and struct.unpack_from("<i", raw, 16)[0] == 16 * 7
    assert len(raw) == 4 + 8 + 4 + 4 + 16 * 7 + 4
    e, w = edxio.read_eigvec(p, 7)
    assert e == -3.25 and np.array_equal(v, w)
    with pytest.raises(edxio.EdxInputError):
        edxio.read_eigvec(p, 8)


def test_output_formats(tmp_path):
    p = str(tmp_path / "eigvals.dat")
    edxio.write_eigvals(p, [-12.3456789012345, 0.5])
    lines = open(p).read().splitlines()
    assert lines[0] == "    1      -12.3456789012"
    assert lines[1] == "    2        0.5000000000"
    p = str(tmp_path / "xas_poles.1")
    edxio.write_poles(p, 2, [1.0, -2.0], [0.5, 1e-12], 3.0, -7.5)
    txt = open(p).read().splitlines()
    assert txt[0] == "#number_of_poles:            2"
    assert txt[1] == "#enegry:                   -7.5000000000"
    assert txt[2] == "#normalization:             3.0000000000"
    pd = edxio.read_poles([p])
    assert pd["npoles"] == [2] and pd["alpha"][0] == [1.0, -2.0] and pd["eigval"][0] == -7.5
    dm = np.zeros((1, 2, 2), dtype=complex)
    dm[0, 0, 1] = 0.25 - 0.5j
    edxio.write_denmat(str(tmp_path / "denmat.dat"), dm)
    d = np.loadtxt(str(tmp_path / "denmat.dat"))
    assert d.shape == (4, 5) and d[1].tolist() == [1, 1, 2, 0.25, -0.5]


# ---- C ABI ----------------------------------------------------------------------------

def _header_functions():
    txt = open(os.path.join(ROOT, "include", "edx.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(edx_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_header_symbol():
    import ctypes
    from edrixs_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from edrixs_b200 import build
        build.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    # the binding declares every header function and nothing else
    assert set(_lib.exported_symbols()) <= set(names)
    assert L.edx_abi_version() == 7


def test_abi_error_path_without_gpu():
    """Host-side validation fails with a status and a message; nothing aborts."""
    import ctypes
    from edrixs_b200 import _lib
    L = _lib.load()
    n = ctypes.c_int64(0)
    assert L.edx_fock_count(20, 10, ctypes.byref(n)) == 0 and n.value == 184756
    assert L.edx_fock_count(70, 10, ctypes.byref(n)) == 1
    assert b"norb" in L.edx_last_error()
    with pytest.raises(_lib.EdxError):
        _lib.call("edx_fock_count", -1, 0, ctypes.byref(n))


def _no_cuda_device():
    try:
        import torch
        return not torch.cuda.is_available()
    except ImportError:
        return True


@pytest.mark.skipif(not _no_cuda_device(), reason="host-validation test; runs where no GPU is visible")
def test_every_entry_point_rejects_null_arguments():
    """The reference STOPs on bad input (src/io.f90:37-39); every libedx entry point instead
    returns EDX_ERR_INVALID with a message, here for an argument list of NULLs and zeros."""
    import ctypes
    from edrixs_b200 import _lib
    _lib.load()
    raw = ctypes.CDLL(_lib.LIB_PATH)          # no argtypes: zeros in every slot
    raw.edx_last_error.restype = ctypes.c_char_p
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "edx.h")).read(), flags=re.S)
    entries = re.findall(r"^int (edx_\w+)\s*\((.*?)\);", txt, flags=re.M | re.S)
    checked = 0
    for name, params in entries:
        nargs = len([p for p in params.split(",") if p.strip() and p.strip() != "void"])
        if nargs == 0:
            continue
        rc = getattr(raw, name)(*([None] * nargs))
        assert rc == 1, (name, rc)
        assert raw.edx_last_error(), name
        checked += 1
    assert checked >= 27


@pytest.mark.skipif(not _no_cuda_device(), reason="host-validation test; runs where no GPU is visible")
def test_matrix_descriptors_are_validated_on_the_host():
    import ctypes
    from edrixs_b200 import _lib
    L = _lib.load()
    nbytes = ctypes.c_size_t(0)
    A = _lib.Csr(nrows=-5, ncols=10, nnz=0)
    assert L.edx_spmm(ctypes.byref(A), 1, 0, None, 1, None, 1, 1.0, 0, 0, 0, 0, 0, 0, None) == 1
    assert b"negative" in L.edx_last_error()
    A = _lib.Csr(nrows=5, ncols=5, nnz=3)
    assert L.edx_spmm(ctypes.byref(A), 1, 0, None, 1, None, 1, 1.0, 0, 0, 0, 0, 0, 0, None) == 1
    assert b"row pointers" in L.edx_last_error()
    assert L.edx_pack_workspace(ctypes.byref(A), ctypes.byref(nbytes)) == 1
    assert L.edx_krylov_workspace(100, 0, None, 10, ctypes.byref(nbytes)) == 1
    assert L.edx_krylov_workspace(-1, 4, None, 10, ctypes.byref(nbytes)) == 1
    assert L.edx_krylov_workspace(100, 4, None, 10, ctypes.byref(nbytes)) == 0 and nbytes.value > 0
    n = ctypes.c_int64(0)
    assert L.edx_fock_count(63, 31, ctypes.byref(n)) == 0 and n.value == 916312070471295267  # C(63,31)
    assert L.edx_fock_count(0, 0, ctypes.byref(n)) == 0 and n.value == 1
    assert L.edx_fock_count(64, 32, ctypes.byref(n)) == 1
    assert L.edx_fock_count(10, 11, ctypes.byref(n)) == 1


# ---- workload generator ------------------------------------------------------------------

def test_siam_seeded_and_hermitian():
    a = siam.make_siam(10, 10, seed=3)
    b = siam.make_siam(10, 10, seed=3)
    assert np.array_equal(a.emat_i, b.emat_i)
    assert np.allclose(a.emat_i, a.emat_i.conj().T)
    assert np.allclose(a.emat_n, a.emat_n.conj().T)
    hop = siam.nonzero_terms(a.emat_i)
    coul = siam.nonzero_terms(a.umat_i)
    assert len(coul[1]) == 340  # the reference's d-shell Slater tensor has 340 nonzeros
    assert len(hop[1]) > 200
    c = siam.make_siam(10, 10, seed=4)
    assert not np.array_equal(a.emat_i, c.emat_i)


def test_fock_states_sorted():
    s = siam.fock_states(8, 3)
    assert len(s) == 56 and np.all(np.diff(s.astype(np.int64)) > 0)
    assert all(bin(int(x)).count("1") == 3 for x in s)


# ---- serving admission (host logic only) ------------------------------------------------

def test_admission_estimates_and_oversize_rejection():
    from concurrent.futures import Future
    from edrixs_b200.serve import ModelSpec, Request, Server, estimate_bytes
    small = Request("rixs", ModelSpec(2, 3, 1), ngs=2, omegas=np.zeros(4), eloss=np.zeros(10), pols=(0, 3))
    big = Request("rixs", ModelSpec(16, 13, 1), ngs=3, omegas=np.zeros(64), eloss=np.zeros(10), pols=(0, 1, 2, 3))
    assert 0 < estimate_bytes(small, True) < estimate_bytes(small, False) < estimate_bytes(big, False)
    srv = Server(hbm_budget=1e9)          # not started: submit() only runs admission checks
    f = srv.submit(big)
    assert isinstance(f, Future) and isinstance(f.exception(timeout=1), MemoryError)
    f2 = srv.submit(small)
    assert not f2.done() and len(srv.waiting) == 1


def test_product_package_never_imports_the_oracle():
    """The oracle is test infrastructure: no module of the product package imports it, so no
    product call can route through it (bench.py's CPU-baseline leg and smoke()'s result check are
    the only other importers)."""
    import ast
    pkg = os.path.join(ROOT, "edrixs_b200")
    offenders = []
    for dirpath, dirnames, filenames in os.walk(pkg):
        dirnames[:] = [d for d in dirnames if not d.startswith("_build")]
        for fn in filenames:
            if not fn.endswith(".py"):
                continue
            path = os.path.join(dirpath, fn)
            tree = ast.parse(open(path).read(), filename=path)
            for node in ast.walk(tree):
                names = []
                if isinstance(node, ast.Import):
                    names = [a.name for a in node.names]
                elif isinstance(node, ast.ImportFrom) and node.module:
                    names = [node.module]
                if any(n == "oracle" or n.startswith("oracle.") for n in names):
                    offenders.append(os.path.relpath(path, ROOT))
    assert not offenders, offenders


def test_device_basis_rejects_unsorted_states():
    """Checked on the host before any device work: the column search needs ascending states."""
    from edrixs_b200 import device
    for bad in ([3, 1, 2], [1, 1]):
        with pytest.raises(ValueError, match="ascending"):
            device.basis_from_states(np.array(bad, dtype=np.uint64))


@pytest.mark.parametrize("body,msg", [
    ("neval=abc", "bad value for neval"), ("eigval_tol=x", "bad value for eigval_tol"),
    ("neval=2.5", "not an integer"), ("num_val_orbs=-3", "must not be negative"),
])
def test_config_bad_values_raise_input_errors(tmp_path, body, msg):
    p = tmp_path / "config.in"
    p.write_text(f"&control\n{body}\n&end\n")
    with pytest.raises(edxio.EdxInputError, match=msg):
        edxio.read_config(str(p))


def test_truncated_eigvec_raises_input_error(tmp_path):
    p = tmp_path / "eigvec.1"
    edxio.write_eigvec(str(p), -1.0, np.ones(4, dtype=np.complex128))
    raw = p.read_bytes()
    for cut in (6, 20, len(raw) - 2):
        p.write_bytes(raw[:cut])
        with pytest.raises(edxio.EdxInputError):
            edxio.read_eigvec(str(p), 4)


def test_unknown_ed_solver_is_refused_above_min_ndim():
    """src/ed_driver.f90:127-171 has branches for ed_solver 0, 1 and 2 only (below min_ndim
    it switches to 0 itself)."""
    from types import SimpleNamespace
    from edrixs_b200 import fedrixs
    cfg = dict(edxio.CONFIG_DEFAULTS, ed_solver=3, min_ndim=1000, ncv=3)
    with pytest.raises(edxio.EdxInputError, match="ed_solver"):
        fedrixs.ed_core(cfg, SimpleNamespace(nrows=5000))
