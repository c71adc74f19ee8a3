"""The in-memory ground-state search over N against the reference's own search loop
(ed_siam_fort with do_ed=0, edrixs/solvers.py:2156-2233), recorded in tests/golden/search_gs.

The recording answered each of the reference's ed_fsolver calls with the oracle (dense
eigensolver, density matrix) through eigvals.dat / denmat.dat.  Here the same oracle answers
solve(N) directly, so what is compared is the walk over N, the choice of the ground-state
occupancy and the two files the search writes.  The device solver (search.device_solver)
builds on the ED core of the drop-in ed_fsolver."""
import json
import os

import numpy as np

from edrixs_b200 import io as edxio
from edrixs_b200 import search
from oracle import pyoracle as orc

NTOT_V, V_NORB = 12, 6


def _oracle_solver(d):
    hop = orc.read_terms(os.path.join(d, "hopping_i.in"), 2)
    coul = orc.read_terms(os.path.join(d, "coulomb_i.in"), 4)
    calls = []

    def solve(N):
        calls.append(N)
        fock = orc.fock_full_N(NTOT_V, N)
        H = orc.build_csr("ham_i", fock, hop, coul, num_val_orbs=NTOT_V)
        e, v = np.linalg.eigh(H.dense())
        dm = orc.denmat(fock, NTOT_V, v[:, 0])
        return search.file_rounded(e[0]), search.impurity_occupancy(dm, V_NORB)

    return solve, calls


def test_search_walks_n_like_the_reference(golden_dir, tmp_path):
    d = os.path.join(golden_dir, "search_gs")
    ref = json.load(open(os.path.join(d, "calls.json")))
    solve, calls = _oracle_solver(d)
    r = search.search_occupancy(NTOT_V, solve, directory=str(tmp_path))
    # the reference's last call is the final ED at the chosen occupancy, outside the search
    assert calls == ref["n_per_call"][:-1]
    assert r.noccu_gs == ref["noccu_gs"] == ref["n_per_call"][-1]
    assert abs(r.eval_gs - ref["eval_i"][0]) < 1e-12
    for fn in ("search_result.dat", "search_gs.log"):
        assert open(os.path.join(tmp_path, fn)).read() == open(os.path.join(d, fn)).read(), fn
    # the last call ran at the chosen occupancy with the caller's settings (solvers.py:2247-2252)
    cfg = edxio.read_config(os.path.join(d, "config_last.in"))
    assert cfg["neval"] == 2 and cfg["ed_solver"] == 2


def test_search_direction_rules_on_synthetic_energies():
    """solvers.py:2181-2225 on energies chosen to exercise each branch: an upward step that
    improves closes the downward direction; a tie counts as an improvement (`eigval >
    eval_gs` is false); the walk stops at the ends of the occupancy range."""
    def run(ntot_v, energy):
        seen = []

        def solve(N):
            seen.append(N)
            return float(energy(N)), 0.0
        return search.search_occupancy(ntot_v, solve), seen

    r, seen = run(8, lambda N: -N)                        # keeps going up to N = 8
    assert seen == [4, 5, 6, 7, 8] and r.noccu_gs == 8
    r, seen = run(8, lambda N: N)                         # first up fails, then down to 0
    assert seen == [4, 5, 3, 2, 1, 0] and r.noccu_gs == 0
    r, seen = run(8, lambda N: (N - 4) ** 2)              # minimum at the start: one step each way
    assert seen == [4, 5, 3] and r.noccu_gs == 4
    r, seen = run(8, lambda N: 0.0 if N in (4, 5) else 1.0)   # tie with the start moves up
    assert seen == [4, 5, 6] and r.noccu_gs == 5
    r, seen = run(7, lambda N: abs(N - 1))                # odd ntot_v: start at 3, down to 1
    assert seen == [3, 4, 2, 1, 0] and r.noccu_gs == 1
    assert [x[0] for x in r.results] == [1, 2, 0, 3, 4]
