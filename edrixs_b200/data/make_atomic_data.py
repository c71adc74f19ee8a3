"""Capture the atomic input tensors of the reference's physics layer as a data file.

The ED/XAS/RIXS hot path consumes one-body (``emat``) and two-body (``umat``) tensors,
dipole transition operators and photon polarisation vectors.  Those come from the
reference's input-generation layer (``edrixs/coulomb_utensor.py:373`` get_umat_slater,
``edrixs/soc.py:6`` atom_hsoc, ``edrixs/photon_transition.py:61`` get_trans_oper,
``edrixs/photon_transition.py:395`` dipole_polvec_rixs, ``:475`` dipole_polvec_xas,
``edrixs/angular_momentum.py:597`` cf_cubic_d), which is outside the hot path.  This
script imports that layer once (a ``matplotlib`` stub stands in for the plotting
dependency) and stores the tensors it returns, so that the seeded workload generator in
``edrixs_b200/siam.py`` runs on machines that do not have the reference installed.

Everything stored is linear in its physical parameter, so unit tensors are kept:
``U(F0,F2,...) = sum_k F_k * U_k`` and ``hsoc(zeta) = zeta * hsoc(1)``.

Usage: ``python edrixs_b200/data/make_atomic_data.py /path/to/edrixs-reference``
"""
import os
import sys
import types

import numpy as np


def _import_reference(path):
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.path.insert(0, path)
    import edrixs  # noqa: E402
    return edrixs


def _sparse4(u, tol=1e-14):
    idx = np.argwhere(np.abs(u) > tol).astype(np.int16)
    return idx, u[tuple(idx.T)].astype(np.complex128)


def main(ref_path, out_path):
    ed = _import_reference(ref_path)
    names = ed.slater_integrals_name(("d", "p"), ("v", "c"))
    data = {"slater_names_dp": np.array(names)}
    for k in range(len(names)):
        unit = np.zeros(len(names))
        unit[k] = 1.0
        idx, val = _sparse4(ed.get_umat_slater("dp", *unit))
        data[f"umat_dp_unit{k}_idx"] = idx
        data[f"umat_dp_unit{k}_val"] = val
    # single d shell (10 orbitals) used by the known-answer ED case
    for k in range(3):
        unit = np.zeros(3)
        unit[k] = 1.0
        idx, val = _sparse4(ed.get_umat_slater("d", *unit))
        data[f"umat_d_unit{k}_idx"] = idx
        data[f"umat_d_unit{k}_val"] = val
    data["hsoc_d_unit"] = ed.atom_hsoc("d", 1.0)
    data["hsoc_p_unit"] = ed.atom_hsoc("p", 1.0)
    data["trans_oper_dp"] = ed.get_trans_oper("dp")
    data["cf_cubic_d_unit"] = ed.cf_cubic_d(1.0)
    # scattering geometry: thin=15 deg, thout=75 deg, phi=0; linear pi (0) / sigma (pi/2)
    thin, thout, phi = np.radians(15.0), np.radians(75.0), 0.0
    pols = [(0.0, 0.0), (0.0, np.pi / 2), (np.pi / 2, 0.0), (np.pi / 2, np.pi / 2)]
    ei, ef = [], []
    for a, b in pols:
        e_in, e_out = ed.dipole_polvec_rixs(thin, thout, phi, a, b, None, ("linear", "linear"))
        ei.append(e_in)
        ef.append(e_out)
    data["rixs_polvec_in"] = np.array(ei, dtype=np.complex128)
    data["rixs_polvec_out"] = np.array(ef, dtype=np.complex128)
    data["rixs_pol_angles"] = np.array(pols)
    data["xas_polvec"] = np.array([ed.dipole_polvec_xas(thin, phi, a) for a in (0.0, np.pi / 2)],
                                  dtype=np.complex128)
    data["geometry_thin_thout_phi"] = np.array([thin, thout, phi])
    np.savez_compressed(out_path, **data)
    print("wrote", out_path, {k: np.shape(v) for k, v in data.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python edrixs_b200/data/make_atomic_data.py /path/to/edrixs-reference")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "atomic_dp.npz")
    main(sys.argv[1], out)
