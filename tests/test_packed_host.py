"""Host side of the packed form and the launch-shape candidates (no GPU needed)."""
import numpy as np
import torch


def _words(cols, idx, vbits):
    w = (np.asarray(cols, dtype=np.uint64) << np.uint64(vbits)) | np.asarray(idx, dtype=np.uint64)
    return torch.from_numpy(w.astype(np.uint32).view(np.int32))


def test_unpack_narrow_and_wide():
    from edrixs_b200.device import PackedMatrix
    vals = torch.tensor([1 + 2j, -3.5, 0.25j], dtype=torch.complex128)
    rp = torch.tensor([0, 2, 3], dtype=torch.int64)
    cols, idx = [1, (1 << 22) - 1], [2, 0]
    cols.append(0)
    idx.append(1)
    diag = torch.zeros(2, dtype=torch.complex128)
    narrow = PackedMatrix(rp, _words(cols, idx, 10), vals, diag, 10)
    r, c, v = narrow.unpack()
    assert c.tolist() == cols and torch.equal(v, vals[idx])
    wide = PackedMatrix(rp, torch.from_numpy(np.asarray(cols, dtype=np.uint32).view(np.int32)), vals, diag, 0,
                        torch.from_numpy(np.asarray(idx, dtype=np.uint16).view(np.int16)))
    r, c, v = wide.unpack()
    assert wide.wide and c.tolist() == cols and torch.equal(v, vals[idx])
    assert wide.nbytes() == narrow.nbytes() + 3 * 2


def test_launch_shape_candidates():
    from edrixs_b200 import tune
    c6 = tune.candidates(6)
    assert {c["col_group"] for c in c6} == {6, 8}
    assert all(c["tiles"] == 1 for c in c6)
    c768 = tune.candidates(768)
    assert {c["col_group"] for c in c768} == {32, 16}
    assert {c["tiles"] for c in c768 if c["col_group"] == 32} == {1, 2, 4}
    assert all(c["threads"] * c["blocks_per_sm"] <= 2048 for c in c6 + c768)
