"""Host side of the tiled layout: the Fock-state tiling that picks row and column tiles.

The tiles are runs of consecutive states that share their high orbitals; for the SIAM
bases (impurity orbitals in the low bits) a row tile is one bath occupation.
"""
import numpy as np
import torch

from oracle import pyoracle as orc


def test_fock_tiles_are_runs_of_shared_high_bits():
    from edrixs_b200 import device
    s = orc.fock_full_N(20, 10)
    st = torch.from_numpy(s)
    for m, p in ((device.TILE_ROWS_MAX, 10), (device.TILE_COLS_MAX, 9)):
        t = device.fock_tiles(st, m).numpy()
        assert t.dtype == np.int32 and t[0] == 0 and t[-1] == len(s)
        assert np.diff(t).max() <= m and np.diff(t).min() >= 1
        key = s >> p
        assert np.array_equal(np.flatnonzero(np.diff(key)) + 1, t[1:-1])


def test_fock_tiles_any_ascending_list():
    from edrixs_b200 import device
    rng = np.random.default_rng(0)
    st = np.unique(rng.integers(0, 1 << 40, size=5000))
    t = device.fock_tiles(torch.from_numpy(st), 128).numpy()
    assert t[0] == 0 and t[-1] == len(st) and np.diff(t).max() <= 128
    # the next larger shift would have produced a run longer than 128
    p = next(q for q in range(64) if np.array_equal(np.flatnonzero(np.diff(st >> q)) + 1, t[1:-1]))
    assert np.diff(np.r_[0, np.flatnonzero(np.diff(st >> (p + 1))) + 1, len(st)]).max() > 128
