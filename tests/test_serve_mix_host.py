"""Host side of the serving benchmark: the seeded request mix (no GPU needed)."""
import math
import types

import numpy as np


def test_serve_mix_is_seeded_and_in_range():
    import bench
    from edrixs_b200 import siam
    args = types.SimpleNamespace(serve_seed=7, serve_requests=48, serve_rate=50.0)
    a, b = bench.serve_mix(args), bench.serve_mix(args)
    assert [(t, r.kind, r.model) for t, r in a] == [(t, r.kind, r.model) for t, r in b]
    times = np.array([t for t, _ in a])
    assert np.all(np.diff(times) > 0) and times[-1] < 48 / 50.0 * 3
    npol_xas = len(siam.atomic()["xas_polvec"])
    for _, r in a:
        norb = 10 + r.model.nbath
        assert 16 <= norb <= 22 and abs(r.model.nelec - norb // 2) <= 1
        assert r.kind in ("ed", "xas", "rixs")
        if r.kind == "xas":
            assert 0 <= r.pols[0] < npol_xas
        if r.kind == "rixs":
            assert all(0 <= p < 4 for p in r.pols) and len(r.omegas) == 8
        assert math.comb(norb, r.model.nelec) <= 705432
    kinds = {r.kind for _, r in a}
    assert kinds == {"ed", "xas", "rixs"}
