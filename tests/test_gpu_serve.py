"""Serving loop: a request's result is the same alone and in a concurrent mix (with
coalescing, other Hamiltonians and other job kinds in flight), within 1e-6 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_alone_vs_mix(cuda):
    from edrixs_b200.serve import ModelSpec, Request, Server
    m1 = ModelSpec(2, 3, 11)
    m2 = ModelSpec(4, 5, 12)
    eloss = np.linspace(-0.5, 8.0, 400)

    def rixs_req(oms):
        return Request("rixs", m1, ngs=2, omegas=np.asarray(oms), eloss=eloss, gamma_c=0.6, gamma_f=0.1,
                       pols=(0, 3), nkryl=60)

    srv = Server(hbm_budget=40e9, workers=3).start()
    try:
        alone_a = srv.submit(rixs_req([0.5, 2.0])).result(timeout=600)
        alone_d = srv.submit(rixs_req([1.0, 4.0, 6.0])).result(timeout=600)
        # the mix: same requests again + an ED on another Hamiltonian + an XAS on the same one
        futs = [srv.submit(rixs_req([0.5, 2.0])), srv.submit(Request("ed", m2, ngs=3)),
                srv.submit(Request("xas", m1, ngs=2, eloss=np.linspace(-3, 12, 300), gamma_c=0.3, pols=(0,),
                                   nkryl=80)),
                srv.submit(rixs_req([1.0, 4.0, 6.0]))]
        mix = [f.result(timeout=600) for f in futs]
    finally:
        srv.shutdown()
    assert rel_linf(mix[0]["spectra"], alone_a["spectra"]) < 1e-6
    assert rel_linf(mix[3]["spectra"], alone_d["spectra"]) < 1e-6
    assert len(mix[1]["eigvals"]) == 3 and np.all(np.diff(mix[1]["eigvals"]) >= 0)
    assert mix[2]["spectrum"].shape == (300,) and np.all(np.isfinite(mix[2]["spectrum"]))
    summ = srv.latency_summary()
    assert summ["n"] == 6 and summ["p99_ms"] >= summ["p50_ms"] > 0


def test_coalesced_requests_match_alone(cuda):
    """Requests that wait while the only worker is busy join one solve: RIXS with different
    ground-state counts, polarisations and incident energies, and XAS with different
    polarisations.  Each gets the result it gets alone, within 1e-6."""
    from edrixs_b200.serve import ModelSpec, Request, Server
    m1 = ModelSpec(2, 3, 21)
    eloss = np.linspace(-0.5, 8.0, 400)

    def rixs_req(oms, ngs, pols):
        return Request("rixs", m1, ngs=ngs, omegas=np.asarray(oms), eloss=eloss, gamma_c=0.6, gamma_f=0.1,
                       pols=pols, nkryl=60)

    def xas_req(pol, ngs):
        return Request("xas", m1, ngs=ngs, eloss=np.linspace(-3, 12, 300), gamma_c=0.3, pols=(pol,), nkryl=80)

    reqs = [lambda: rixs_req([0.5, 2.0], 1, (1,)), lambda: rixs_req([1.0, 2.0, 6.0], 2, (0, 3)),
            lambda: xas_req(0, 1), lambda: xas_req(1, 2)]
    srv = Server(hbm_budget=40e9, workers=1).start()
    try:
        alone = [srv.submit(f()).result(timeout=600) for f in reqs]
        # keep the one worker busy, then queue all four: they wait and are grouped
        busy = srv.submit(Request("ed", ModelSpec(6, 8, 5), ngs=3))
        futs = [srv.submit(f()) for f in reqs]
        busy.result(timeout=600)
        mix = [f.result(timeout=600) for f in futs]
    finally:
        srv.shutdown()
    assert mix[0]["coalesced"] == 2 and mix[2]["coalesced"] == 2
    for a, b in zip(alone[:2], mix[:2]):
        assert b["spectra"].shape == a["spectra"].shape
        assert rel_linf(b["spectra"], a["spectra"]) < 1e-6
    for a, b in zip(alone[2:], mix[2:]):
        assert rel_linf(b["spectrum"], a["spectrum"]) < 1e-6


def test_failed_request_does_not_stop_server(cuda):
    from edrixs_b200.serve import ModelSpec, Request, Server
    srv = Server(hbm_budget=40e9, workers=2).start()
    try:
        bad = srv.submit(Request("xas", ModelSpec(2, 3, 1), ngs=1, eloss=np.linspace(0, 1, 10), pols=(7,)))
        with pytest.raises(Exception):
            bad.result(timeout=300)
        ok = srv.submit(Request("ed", ModelSpec(2, 3, 1), ngs=2)).result(timeout=300)
        assert len(ok["eigvals"]) == 2
    finally:
        srv.shutdown()


def test_slab_only_residents_match_packed(cuda, monkeypatch):
    """Intermediate sectors above serve.SLAB_ONLY_ROWS are held in the slab form alone (no CSR
    built), with the absorption edge from a plain Lanczos run.  With the threshold at 0 the
    same XAS and RIXS requests give the results of the packed residents within 1e-6."""
    from edrixs_b200 import device, serve
    from edrixs_b200.serve import ModelSpec, Request, Server
    m = ModelSpec(4, 5, 31)
    eloss = np.linspace(-0.5, 8.0, 300)
    reqs = [lambda: Request("rixs", m, ngs=2, omegas=np.array([0.5, 2.5]), eloss=eloss, gamma_c=0.6, gamma_f=0.1,
                            pols=(0, 3), nkryl=60),
            lambda: Request("xas", m, ngs=2, eloss=np.linspace(-3, 12, 300), gamma_c=0.3, pols=(1,), nkryl=80)]
    out = {}
    for thr in (serve.SLAB_ONLY_ROWS, 0):
        monkeypatch.setattr(serve, "SLAB_ONLY_ROWS", thr)
        srv = Server(hbm_budget=40e9, workers=1).start()
        try:
            out[thr] = [srv.submit(f()).result(timeout=600) for f in reqs]
            Hn = srv.residents[m].Hn
        finally:
            srv.shutdown()
        assert isinstance(Hn, device.KronMatrix if thr == 0 else device.PackedMatrix)
    a, b = out[serve.SLAB_ONLY_ROWS], out[0]
    assert rel_linf(b[0]["spectra"], a[0]["spectra"]) < 1e-6
    assert rel_linf(b[1]["spectrum"], a[1]["spectrum"]) < 1e-6

