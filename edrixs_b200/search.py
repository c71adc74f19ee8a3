"""Ground-state search over the total occupancy N, in memory.

The reference's ``ed_siam_fort(..., do_ed=0)`` (edrixs/solvers.py:2156-2240) finds the
occupancy of the ground state by calling ``ed_fsolver`` once per N with ``ed_solver=1``,
``neval=1``, ``nvector=1``.  Each call writes ``fock_i.in``, runs the Fortran solver, and
reads ``eigvals.dat`` and ``denmat.dat`` back.  Here the hopping and Coulomb terms stay in
memory; each N builds its basis and Hamiltonian on the device and solves it there.

The walk over N is the reference's, step for step:
* start at N0 = ntot_v // 2 (:2161-2176);
* step i = 0 .. ntot_v//2 - 1 tries N0 + i + 1 while the upward direction is open, then
  N0 - i - 1 while the downward one is open (:2181-2225).  An energy above the best so far
  closes that direction.  An energy at or below it becomes the best and closes the other
  direction;
* the impurity occupancy of each N is the trace of the first ``v_norb`` diagonal entries of
  the density matrix of its lowest state (:2177,2199,2221);
* the reference decides on the numbers it reads back from eigvals.dat and denmat.dat, which
  carry 10 decimals (f20.10, src/io.f90:587-635).  ``file_rounded`` applies the same round
  trip, so that near-ties between occupancies go the same way;
* the results are sorted by energy (:2229).  ``search_result.dat`` holds them as
  ``{:10d}{:20.10f}{:20.10f}`` (:2230-2232) and ``search_gs.log`` in the order visited
  (:2178,2200,2222).

The caller's last step (:2235-2262: shift the levels by c_level and solve again at the
ground-state occupancy with the requested neval/nvector) is an ordinary ED call; it is not
part of the search.
"""
import os
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Tuple

import numpy as np


def file_rounded(x):
    """A value after the f20.10 write and the np.loadtxt read of the reference's files."""
    return float("{:20.10f}".format(float(x)))


def impurity_occupancy(denmat0, v_norb):
    """Trace over the first v_norb orbitals of one density matrix, from the entries as
    denmat.dat carries them and summed as the reference sums them: numpy's sum over the
    complex diagonal (edrixs/solvers.py:2174-2177), whose pairwise order can differ from a
    left-to-right sum in the last bit."""
    diag = np.array([complex(file_rounded(denmat0[i, i].real), file_rounded(denmat0[i, i].imag))
                     for i in range(v_norb)])
    return float(np.sum(diag).real)


@dataclass
class SearchResult:
    noccu_gs: int
    eval_gs: float
    visited: List[Tuple[int, float, float]]          # (N, E_0(N), impurity occupancy), in order visited
    results: List[Tuple[int, float, float]] = field(default_factory=list)  # the same, sorted by energy


def device_solver(hopping, coulomb, ntot_v, v_norb, *, maxiter=1000, eigval_tol=1e-8, min_ndim=1000):
    """solve(N) -> (E_0, impurity occupancy) on the current CUDA device: Fock basis, H_i build,
    lowest eigenpair (the ED core of ed_fsolver with ed_solver=1, neval=nvector=1) and the
    density matrix of that eigenvector."""
    from . import device
    from .fedrixs import ed_core
    device.require_cuda()
    cfg = {"ed_solver": 1, "neval": 1, "nvector": 1, "maxiter": maxiter, "eigval_tol": eigval_tol,
           "min_ndim": min_ndim}

    def solve(N):
        basis = device.fock_unrank(ntot_v, N)
        H = device.build_csr(device.HAM_I, basis, hopping, coulomb, num_val_orbs=ntot_v)
        e, v = ed_core(cfg, H)
        dm = device.denmat(basis, ntot_v, v).cpu().numpy()
        return file_rounded(e[0]), impurity_occupancy(dm[0], v_norb)

    return solve


def search_occupancy(ntot_v, solve: Callable[[int], Tuple[float, float]], *,
                     directory: Optional[str] = None) -> SearchResult:
    """Walk N from ntot_v // 2 as edrixs/solvers.py:2156-2233 does.  solve(N) returns the
    lowest energy at N and its impurity occupancy (``device_solver`` builds one).  With
    ``directory``, search_gs.log and search_result.dat are written there."""
    visited = []
    n0 = ntot_v // 2
    eval_gs, occ = solve(n0)
    noccu_gs = n0
    visited.append((n0, eval_gs, occ))
    up, down = True, True
    for i in range(ntot_v // 2):
        if up:
            n = n0 + i + 1
            e, occ = solve(n)
            if e > eval_gs:
                up = False
            else:
                down = False
                eval_gs, noccu_gs = e, n
            visited.append((n, e, occ))
        if down:
            n = n0 - i - 1
            e, occ = solve(n)
            if e > eval_gs:
                down = False
            else:
                up = False
                eval_gs, noccu_gs = e, n
            visited.append((n, e, occ))
    results = sorted(visited, key=lambda x: x[1])
    if directory is not None:
        with open(os.path.join(directory, "search_gs.log"), "w") as f:
            for n, e, o in visited:
                print(n, e, o, file=f)
        with open(os.path.join(directory, "search_result.dat"), "w") as f:
            for n, e, o in results:
                f.write("{:10d}{:20.10f}{:20.10f}\n".format(n, e, o))
    return SearchResult(noccu_gs, eval_gs, visited, results)
