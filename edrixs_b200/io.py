"""File formats of the ED/XAS/RIXS drop-in boundary.

The reference's Fortran core exchanges everything with its Python callers through files in
the working directory.  This module reads and writes exactly those formats:

inputs (read by the solvers; written by the reference's Python layer)
  config.in          Fortran namelist ``&control ... &end`` (src/io.f90:2-67, defaults at
                     :17-32; writer edrixs/iostream.py:238-276).  Any subset of keys, any
                     order, ``1E-10``/``1d-10`` and ``.true.``/``T`` are accepted.
  hopping_*.in       count, then ``i j re im`` (1-based) per line (src/io.f90:70-117;
                     writer edrixs/iostream.py:165-198, empty operator = ``1 1 0 0``)
  coulomb_*.in       count, then ``i j k l re im`` (src/io.f90:120-170; writer :201-235)
  fock_*.in          ndim, then one decimal Fock state per line (src/io.f90:174-361;
                     writer edrixs/fock_basis.py:398-451)
  transop_*.in       as hopping (src/io.f90:364-512)
  eigvec.N           Fortran unformatted sequential: record(eigval f64), record(c128[n])
                     (src/io.f90:544-584)
outputs (written by the solvers; read by the reference's Python layer)
  eigvals.dat        ``(i5, f20.10)`` (src/io.f90:587-607)
  denmat.dat         ``(3i5, 2f20.10)`` as (vector, i, j, re, im) (src/io.f90:610-635)
  xas_poles.N /      ``(a20, i10)`` number of poles, ``(a20, f20.10)`` energy and
  rixs_poles.N       normalization, then ``(i5, 2f20.10)`` (src/io.f90:515-541)
  opavg.dat          ``(1i5, 4f20.10)`` (src/io.f90:638-659)
"""
import os
import re
import struct

import numpy as np

# src/io.f90:17-32 defaults of the namelist
CONFIG_DEFAULTS = {
    "ed_solver": 1, "num_val_orbs": 2, "num_core_orbs": 2, "neval": 1, "nvector": 1,
    "idump": False, "num_gs": 1, "maxiter": 500, "linsys_max": 500, "min_ndim": 1000,
    "ncv": None, "eigval_tol": 1e-8, "linsys_tol": 1e-8, "nkryl": 500, "omega_in": 0.0,
    "gamma_in": 0.1,
}
_INT_KEYS = {"ed_solver", "num_val_orbs", "num_core_orbs", "neval", "nvector", "num_gs",
             "maxiter", "linsys_max", "min_ndim", "ncv", "nkryl"}
_FLOAT_KEYS = {"eigval_tol", "linsys_tol", "omega_in", "gamma_in"}
_BOOL_KEYS = {"idump"}


class EdxInputError(RuntimeError):
    """A required input file is missing or malformed (the reference STOPs here)."""


def _need(path):
    if not os.path.exists(path):
        raise EdxInputError(f"fedrixs >>> ERROR: {os.path.basename(path)} doesn't exist")


def _fortran_float(tok):
    return float(tok.lower().replace("d", "e"))


def _fortran_bool(tok):
    t = tok.strip().lower().lstrip(".")
    if t.startswith("t"):
        return True
    if t.startswith("f"):
        return False
    raise EdxInputError(f"bad logical value in config.in: {tok!r}")


def read_config(path="config.in"):
    """Parse the ``&control`` namelist (src/io.f90:2-67)."""
    _need(path)
    with open(path) as f:
        text = f.read()
    m = re.search(r"&control(.*?)(?:&end|/\s*$|/\s*\n)", text, flags=re.S | re.I)
    if m is None:
        raise EdxInputError("config.in: no &control namelist group found")
    body = m.group(1)
    # strip Fortran comments
    body = "\n".join(line.split("!")[0] for line in body.splitlines())
    cfg = dict(CONFIG_DEFAULTS)
    for key, val in re.findall(r"([A-Za-z_][A-Za-z0-9_]*)\s*=\s*([^,\n]+)", body):
        k = key.lower()
        v = val.strip().rstrip(",").strip()
        try:
            if k in _INT_KEYS:
                x = float(v.lower().replace("d", "e"))
                if not x.is_integer():
                    raise ValueError(f"{v!r} is not an integer")
                cfg[k] = int(x)
            elif k in _FLOAT_KEYS:
                cfg[k] = _fortran_float(v)
            elif k in _BOOL_KEYS:
                cfg[k] = _fortran_bool(v)
            else:
                raise EdxInputError(f"config.in: unknown namelist key {key!r}")
        except ValueError as e:
            raise EdxInputError(f"config.in: bad value for {key}: {e}") from None
    for k in _INT_KEYS:
        if cfg[k] is not None and cfg[k] < 0:
            raise EdxInputError(f"config.in: {k} must not be negative (got {cfg[k]})")
    if cfg["ncv"] is None:  # io.f90:27 ncv = neval + 2 (evaluated after neval's default)
        cfg["ncv"] = CONFIG_DEFAULTS["neval"] + 2
    return cfg


def _count(path, line):
    try:
        n = int(line.split()[0])
    except (ValueError, IndexError):
        raise EdxInputError(f"{path}: the first line must hold the count, got {line.strip()!r}") from None
    if n < 0:
        raise EdxInputError(f"{path}: negative count {n}")
    return n


def _read_counted(path, nidx):
    """Line 1 = count, then `nidx` 1-based orbital indices and a complex value per term
    (src/io.f90:86-152; written by edrixs/iostream.py:165-236)."""
    _need(path)
    with open(path) as f:
        first = f.readline()
        if not first.strip():
            raise EdxInputError(f"{path}: empty file")
        n = _count(path, first)
        data = f.read().split()
    need = n * (nidx + 2)
    if len(data) < need:
        raise EdxInputError(f"{path}: expected {n} terms, file is short")
    arr = np.array(data[:need], dtype=object).reshape(n, nidx + 2)
    try:
        idx = np.array([int(x) for x in arr[:, :nidx].ravel()], dtype=np.int64).reshape(n, nidx)
        vals = np.array([_fortran_float(x) for x in arr[:, nidx:].ravel()], dtype=np.float64)
    except ValueError as e:
        raise EdxInputError(f"{path}: malformed term ({e})") from None
    if n and (idx.min() < 1 or idx.max() > 64):
        raise EdxInputError(f"{path}: orbital indices must lie in 1..64 (1-based)")
    val = vals.reshape(n, 2) @ np.array([1.0, 1j])
    return idx.astype(np.int32), val.astype(np.complex128)


def read_hopping(path):
    """Two-fermion terms (hopping_*.in, transop_*.in) -> (idx int32[n,2] 1-based, val c128)."""
    return _read_counted(path, 2)


def read_coulomb(path):
    """Four-fermion terms (coulomb_*.in) -> (idx int32[n,4] 1-based, val c128)."""
    return _read_counted(path, 4)


def read_fock(path):
    """Fock basis file -> uint64 array (reference keeps int64; values are < 2^63)."""
    _need(path)
    with open(path) as f:
        n = _count(path, f.readline())
        data = f.read().split()
    if len(data) < n:
        raise EdxInputError(f"{path}: expected {n} states, file is short")
    try:
        states = np.array(data[:n], dtype=np.int64)
    except (ValueError, OverflowError) as e:
        raise EdxInputError(f"{path}: malformed state ({e})") from None
    # the writer sorts (edrixs/fock_basis.py:444) and the column search needs it
    # (src/utils.f90:2-40): an unsorted or repeated list would give wrong matrices silently
    if n > 1 and not np.all(np.diff(states) > 0):
        raise EdxInputError(f"{path}: states are not strictly ascending")
    if n and states[0] < 0:
        raise EdxInputError(f"{path}: negative state")
    return states.astype(np.uint64)


def read_eigvec(path, n=None):
    """Fortran unformatted ``eigvec.N`` -> (eigval, c128[n]) (src/io.f90:563-584)."""
    _need(path)
    with open(path, "rb") as f:
        raw = f.read()
    pos = 0
    recs = []
    while pos < len(raw):
        if pos + 4 > len(raw):
            raise EdxInputError(f"{path}: truncated Fortran record")
        (ln,) = struct.unpack_from("<i", raw, pos)
        pos += 4
        if ln < 0 or pos + ln + 4 > len(raw):
            raise EdxInputError(f"{path}: truncated Fortran record")
        recs.append(raw[pos:pos + ln])
        pos += ln
        (ln2,) = struct.unpack_from("<i", raw, pos)
        pos += 4
        if ln2 != ln:
            raise EdxInputError(f"{path}: corrupt Fortran record markers")
    if len(recs) < 2 or len(recs[0]) != 8 or len(recs[1]) % 16:
        raise EdxInputError(f"{path}: not an eigvec file")
    e = struct.unpack("<d", recs[0])[0]
    v = np.frombuffer(recs[1], dtype=np.complex128).copy()
    if n is not None and len(v) != n:
        raise EdxInputError(f"{path}: eigenvector has {len(v)} entries, expected {n}")
    return e, v


def write_eigvec(path, eigval, vec):
    """src/io.f90:544-560 (gfortran sequential unformatted, 4-byte record markers)."""
    vec = np.ascontiguousarray(vec, dtype=np.complex128)
    nb = vec.nbytes
    if nb >= 2**31:
        raise ValueError("eigenvector record exceeds 2 GiB; subrecords are not written")
    with open(path, "wb") as f:
        f.write(struct.pack("<i", 8) + struct.pack("<d", float(eigval)) + struct.pack("<i", 8))
        f.write(struct.pack("<i", nb))
        f.write(vec.tobytes())
        f.write(struct.pack("<i", nb))


def write_eigvals(path, eigvals):
    with open(path, "w") as f:
        for i, e in enumerate(eigvals):
            f.write(f"{i + 1:5d}{e:20.10f}\n")


def write_denmat(path, denmat):
    """denmat: complex (nvector, nv, nv) with [k, i, j] = <c+_i c_j> of vector k."""
    nvec, nv, _ = denmat.shape
    lines = []
    for i in range(nvec):
        d = denmat[i]
        for j in range(nv):
            for k in range(nv):
                lines.append(f"{i + 1:5d}{j + 1:5d}{k + 1:5d}{d[j, k].real:20.10f}{d[j, k].imag:20.10f}\n")
    with open(path, "w") as f:
        f.writelines(lines)


def write_poles(path, neff, alpha, beta, norm, e_gs):
    lines = [f"{'#number_of_poles:':<20s}{neff:10d}\n",
             f"{'#enegry:':<20s}{e_gs:20.10f}\n",
             f"{'#normalization:':<20s}{norm:20.10f}\n"]
    for i in range(neff):
        lines.append(f"{i + 1:5d}{alpha[i]:20.10f}{beta[i]:20.10f}\n")
    with open(path, "w") as f:
        f.writelines(lines)


def read_poles(file_list):
    """Same dict layout as edrixs/iostream.py:279-323 read_poles_from_file."""
    out = {"npoles": [], "eigval": [], "norm": [], "alpha": [], "beta": []}
    for fn in file_list:
        with open(fn) as f:
            neff = int(f.readline().split()[1])
            e = float(f.readline().split()[1])
            nrm = float(f.readline().split()[1])
            a, b = [], []
            for _ in range(neff):
                t = f.readline().split()
                a.append(float(t[1]))
                b.append(float(t[2]))
        out["npoles"].append(neff)
        out["eigval"].append(e)
        out["norm"].append(nrm)
        out["alpha"].append(a)
        out["beta"].append(b)
    return out


def write_opavg(path, eigvals, opavg):
    with open(path, "w") as f:
        for i, (e, o) in enumerate(zip(eigvals, opavg)):
            f.write(f"{i + 1:5d}{e:20.10f}{o.real:20.10f}{o.imag:20.10f}\n")


# ---- writers of the input files (same text the reference's Python layer produces) ----

def write_emat(emat, fname, tol=1e-12):
    """edrixs/iostream.py:165-198: nonzeros of a rank-2 tensor, row-major order."""
    a1, a2 = np.nonzero(np.abs(emat) > tol)
    sp = "    "
    with open(fname, "w") as f:
        if len(a1) == 0:
            f.write("{:10d}\n".format(1))
            f.write("{:10d}{}{:10d}{}{:.15f}{}{:.15f}{}\n".format(1, sp, 1, sp, 0.0, sp, 0.0, sp))
            return
        f.write("{:20d}\n".format(len(a1)))
        for i, j in zip(a1, a2):
            v = emat[i, j]
            f.write("{:10d}{}{:10d}{}{:.15f}{}{:.15f}{}\n".format(i + 1, sp, j + 1, sp, v.real, sp,
                                                                 v.imag, sp))


def write_umat(umat, fname, tol=1e-12):
    """edrixs/iostream.py:201-235: nonzeros of a rank-4 tensor, row-major order."""
    nz = np.nonzero(np.abs(umat) > tol)
    sp = "    "
    with open(fname, "w") as f:
        if len(nz[0]) == 0:
            f.write("{:10d}\n".format(1))
            f.write("".join("{:10d}{}".format(1, sp) for _ in range(4)) +
                    "{:.15f}{}{:.15f}{}\n".format(0.0, sp, 0.0, sp))
            return
        f.write("{:20d}\n".format(len(nz[0])))
        for i, j, k, l in zip(*nz):
            v = umat[i, j, k, l]
            f.write("".join("{:10d}{}".format(x + 1, sp) for x in (i, j, k, l)) +
                    "{:.15f}{}{:.15f}{}\n".format(v.real, sp, v.imag, sp))


def write_config(directory=".", ed_solver=1, num_val_orbs=2, num_core_orbs=2, neval=1, nvector=1,
                 ncv=1, idump=True, num_gs=1, maxiter=500, linsys_max=1000, min_ndim=1000,
                 nkryl=500, eigval_tol=1e-8, linsys_tol=1e-10, omega_in=0.0, gamma_in=0.1):
    """edrixs/iostream.py:238-276 (same keys, same text)."""
    items = ["&control", f"ed_solver={ed_solver}", f"num_val_orbs={num_val_orbs}",
             f"num_core_orbs={num_core_orbs}", f"neval={neval}", f"nvector={nvector}",
             f"ncv={ncv}", "idump=" + (".true." if idump else ".false."), f"num_gs={num_gs}",
             f"maxiter={maxiter}", f"linsys_max={linsys_max}", f"min_ndim={min_ndim}",
             f"nkryl={nkryl}", f"eigval_tol={eigval_tol}", f"linsys_tol={linsys_tol}",
             f"omega_in={omega_in}", f"gamma_in={gamma_in}", "&end"]
    with open(os.path.join(directory, "config.in"), "w") as f:
        f.write("\n".join(items) + "\n")


def write_fock(fname, states):
    """edrixs/fock_basis.py:398-451 layout: ndim, then one decimal per line (ascending)."""
    states = np.asarray(states, dtype=np.uint64)
    with open(fname, "w") as f:
        f.write(f"{len(states)}\n")
        f.write("\n".join(str(int(s)) for s in states))
        f.write("\n")
