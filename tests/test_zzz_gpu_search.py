"""The ground-state search over N with its device solver, against the reference's own search
loop recorded in tests/golden/search_gs (ed_siam_fort with do_ed=0,
edrixs/solvers.py:2156-2233).  Energies and occupancies agree to the 10 decimals the
reference's files carry, give or take one unit in the last place (the device eigensolver
and the oracle round differently in the last bits)."""
import json
import os

import numpy as np
import pytest

from edrixs_b200 import io as edxio
from edrixs_b200 import search


@pytest.mark.gpu
def test_device_search_walks_n_like_the_reference(cuda, golden_dir, tmp_path):
    d = os.path.join(golden_dir, "search_gs")
    ref = json.load(open(os.path.join(d, "calls.json")))
    hop = edxio.read_hopping(os.path.join(d, "hopping_i.in"))
    coul = edxio.read_coulomb(os.path.join(d, "coulomb_i.in"))
    r = search.search_occupancy(12, search.device_solver(hop, coul, 12, 6), directory=str(tmp_path))
    assert [v[0] for v in r.visited] == ref["n_per_call"][:-1]
    assert r.noccu_gs == ref["noccu_gs"]
    ours = np.loadtxt(os.path.join(tmp_path, "search_result.dat"), ndmin=2)
    theirs = np.loadtxt(os.path.join(d, "search_result.dat"), ndmin=2)
    assert ours.shape == theirs.shape
    assert np.array_equal(ours[:, 0], theirs[:, 0])
    assert np.abs(ours[:, 1:] - theirs[:, 1:]).max() <= 2e-10
