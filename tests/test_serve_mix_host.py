"""Host side of the serving benchmark: the seeded request mix (no GPU needed)."""
import math
import types

import numpy as np
import pytest


def test_serve_mix_is_seeded_and_in_range():
    import bench
    from edrixs_b200 import siam
    args = types.SimpleNamespace(serve_seed=7, serve_requests=48, serve_rate=50.0, serve_norb_max=26)
    a, b = bench.serve_mix(args), bench.serve_mix(args)
    assert [(t, r.kind, r.model) for t, r in a] == [(t, r.kind, r.model) for t, r in b]
    times = np.array([t for t, _ in a])
    assert np.all(np.diff(times) > 0) and times[-1] < 48 / 50.0 * 3
    npol_xas = len(siam.atomic()["xas_polvec"])
    for _, r in a:
        norb = 10 + r.model.nbath
        assert 16 <= norb <= 26 and abs(r.model.nelec - norb // 2) <= 1
        assert r.kind in ("ed", "xas", "rixs")
        if r.kind == "xas":
            assert 0 <= r.pols[0] < npol_xas
        if r.kind == "rixs":
            assert all(0 <= p < 4 for p in r.pols) and len(r.omegas) == 8
        assert math.comb(norb, r.model.nelec) <= 10400600
    kinds = {r.kind for _, r in a}
    assert kinds == {"ed", "xas", "rixs"}
    assert {10 + r.model.nbath for _, r in a} >= {16, 26}  # both ends of the stated range
    small = bench.serve_mix(types.SimpleNamespace(serve_seed=7, serve_requests=48, serve_rate=50.0,
                                                  serve_norb_max=22))
    assert max(10 + r.model.nbath for _, r in small) <= 22


def test_coalesce_key_groups_compatible_requests():
    from edrixs_b200.serve import ModelSpec, Request, coalesce_key
    m, m2 = ModelSpec(4, 7, 1), ModelSpec(4, 7, 2)
    el = np.linspace(-0.5, 12.0, 1000)
    a = Request("rixs", m, ngs=1, omegas=np.array([1.0]), eloss=el, pols=(0,))
    b = Request("rixs", m, ngs=3, omegas=np.array([2.0, 3.0]), eloss=el.copy(), pols=(1, 2))
    assert coalesce_key(a) == coalesce_key(b)
    assert coalesce_key(a) != coalesce_key(Request("rixs", m2, omegas=np.array([1.0]), eloss=el))
    assert coalesce_key(a) != coalesce_key(Request("rixs", m, omegas=np.array([1.0]), eloss=el[:500]))
    assert coalesce_key(a) != coalesce_key(Request("rixs", m, omegas=np.array([1.0]), eloss=el, gamma_f=0.3))
    x1 = Request("xas", m, ngs=1, eloss=el, pols=(0,), nkryl=200)
    x2 = Request("xas", m, ngs=2, eloss=el[:10], pols=(1,), nkryl=200)
    assert coalesce_key(x1) == coalesce_key(x2) != coalesce_key(a)
    assert coalesce_key(Request("ed", m)) is None


def test_scheduler_groups_waiting_requests_when_a_worker_frees():
    """The scheduler (no GPU: a fake worker takes the jobs) hands a request to a worker only
    when one is free, and takes every waiting request with the same coalesce_key along."""
    import threading
    import time
    from edrixs_b200.serve import ModelSpec, Request, Server
    srv = Server(hbm_budget=1e12, workers=1)
    groups = []
    release = threading.Event()

    def fake_worker():
        while True:
            job = srv.jobs.get()
            if job is None:
                return
            group, res, need = job
            groups.append([r.id for r, _ in group])
            release.wait(5)
            with srv.cv:
                res.busy -= 1
                srv.inflight_bytes -= need
                srv.free_workers += 1
                srv.cv.notify_all()

    sched = threading.Thread(target=srv._schedule, daemon=True)
    worker = threading.Thread(target=fake_worker, daemon=True)
    sched.start()
    worker.start()
    m, m2 = ModelSpec(4, 7, 1), ModelSpec(4, 7, 2)
    el = np.linspace(-0.5, 12.0, 100)
    first = Request("ed", m2)
    srv.submit(first)
    time.sleep(0.3)  # the one worker now holds the ED job
    a = Request("rixs", m, ngs=1, omegas=np.array([1.0]), eloss=el, pols=(0,))
    x = Request("xas", m, ngs=1, eloss=el, pols=(0,))
    b = Request("rixs", m, ngs=2, omegas=np.array([2.0]), eloss=el, pols=(1,))
    c = Request("rixs", m2, ngs=1, omegas=np.array([2.0]), eloss=el, pols=(1,))
    for r in (a, x, b, c):
        srv.submit(r)
    time.sleep(0.3)
    assert groups == [[first.id]]  # nothing else dispatched while the worker is busy
    release.set()
    deadline = time.time() + 5
    while len(groups) < 4 and time.time() < deadline:
        time.sleep(0.05)
    with srv.cv:
        srv.stop_flag = True
        srv.cv.notify_all()
    srv.jobs.put(None)
    assert groups[1] == [a.id, b.id]  # same Hamiltonian and settings: one solve
    assert sorted(map(tuple, groups[2:])) == sorted([(x.id,), (c.id,)])


def test_cancelled_requests_leave_the_queue_and_the_coalesced_solve():
    """Future.cancel() on a waiting request removes it: it is not dispatched, and the requests
    it would have been coalesced with still run.  A dispatched request can no longer be
    cancelled.  (No GPU: a fake worker takes the jobs.)"""
    import threading
    import time
    from edrixs_b200.serve import ModelSpec, Request, Server
    srv = Server(hbm_budget=1e12, workers=1)
    groups = []
    release = threading.Event()

    def fake_worker():
        while True:
            job = srv.jobs.get()
            if job is None:
                return
            group, res, need = job
            groups.append([r.id for r, _ in group])
            release.wait(5)
            with srv.cv:
                res.busy -= 1
                srv.inflight_bytes -= need
                srv.free_workers += 1
                srv.cv.notify_all()

    sched = threading.Thread(target=srv._schedule, daemon=True)
    worker = threading.Thread(target=fake_worker, daemon=True)
    sched.start()
    worker.start()
    m, m2 = ModelSpec(4, 7, 1), ModelSpec(4, 7, 2)
    el = np.linspace(-0.5, 12.0, 100)
    first = Request("ed", m2)
    f_first = srv.submit(first)
    time.sleep(0.3)
    assert groups == [[first.id]] and not f_first.cancel()   # running: not cancellable
    a = Request("rixs", m, ngs=1, omegas=np.array([1.0]), eloss=el, pols=(0,))
    b = Request("rixs", m, ngs=2, omegas=np.array([2.0]), eloss=el, pols=(1,))
    c = Request("ed", m)
    fa, fb, fc = srv.submit(a), srv.submit(b), srv.submit(c)
    assert fa.cancel() and fc.cancel()
    release.set()
    deadline = time.time() + 5
    while len(groups) < 2 and time.time() < deadline:
        time.sleep(0.05)
    time.sleep(0.3)
    with srv.cv:
        srv.stop_flag = True
        srv.cv.notify_all()
    srv.jobs.put(None)
    assert groups == [[first.id], [b.id]]
    assert fa.cancelled() and fc.cancelled() and fb.running()
    assert srv.waiting == [] and srv.free_workers == 1 and srv.inflight_bytes == 0


def test_shutdown_cancels_waiting_requests_and_refuses_new_ones():
    """After shutdown no future is left pending for ever: waiting requests are cancelled and
    later submissions fail at once.  (Server not started: no GPU.)"""
    from concurrent.futures import CancelledError
    from edrixs_b200.serve import ModelSpec, Request, Server
    srv = Server(hbm_budget=1e12, workers=1)
    f1 = srv.submit(Request("ed", ModelSpec(4, 7, 1)))
    srv.shutdown()
    with pytest.raises(CancelledError):
        f1.result(timeout=1)
    f2 = srv.submit(Request("ed", ModelSpec(4, 7, 2)))
    with pytest.raises(RuntimeError, match="shut down"):
        f2.result(timeout=1)
    assert srv.waiting == []


def test_shutdown_between_pick_and_queue_leaves_no_future_pending():
    """shutdown() that runs while the scheduler hands a picked request to the job queue must
    not strand it: the job is queued ahead of the workers' stop markers, so a worker still
    takes it and its future completes.  The job queue here stalls the scheduler inside its
    put and starts shutdown() meanwhile.  (No GPU: a fake worker takes the jobs.)"""
    import queue
    import threading
    import time
    from edrixs_b200.serve import ModelSpec, Request, Server
    srv = Server(hbm_budget=1e12, workers=1)
    stalled = []

    class StallingQueue(queue.Queue):
        def put(self, item, *a, **kw):
            if item is not None and not stalled:
                t = threading.Thread(target=srv.shutdown, daemon=True)
                stalled.append(t)
                t.start()
                time.sleep(0.3)  # the scheduler is descheduled here; shutdown() runs meanwhile
            super().put(item, *a, **kw)

    srv.jobs = StallingQueue()

    def fake_worker():
        while True:
            job = srv.jobs.get()
            if job is None:
                return
            group, res, need = job
            for r, f in group:
                f.set_result(r.id)
            with srv.cv:
                res.busy -= 1
                srv.inflight_bytes -= need
                srv.free_workers += 1
                srv.cv.notify_all()

    worker = threading.Thread(target=fake_worker, daemon=True)
    worker.start()
    srv.threads.append(worker)
    sched = threading.Thread(target=srv._schedule, daemon=True)
    sched.start()
    req = Request("ed", ModelSpec(4, 7, 1))
    fut = srv.submit(req)
    assert fut.result(timeout=5) == req.id
    stalled[0].join(timeout=5)
    worker.join(timeout=5)
    assert not worker.is_alive() and srv.stop_flag
    assert srv.free_workers == 1 and srv.inflight_bytes == 0


def test_admission_estimate_of_large_models():
    """The admission estimate of the largest models of the serving mix (26 valence
    spin-orbitals) fits the 150 GB budget for ED, XAS and RIXS (slab-only H_n, streamed RIXS),
    and keeps the stored-projection form for small RIXS requests."""
    from edrixs_b200 import serve
    from edrixs_b200.serve import ModelSpec, Request
    big = ModelSpec(16, 13, 1)
    eloss = np.linspace(-0.5, 12.0, 1000)
    reqs = [Request("ed", big, ngs=4), Request("xas", big, ngs=3, eloss=eloss, pols=(0,)),
            Request("rixs", big, ngs=3, omegas=np.linspace(0, 8, 8), eloss=eloss, pols=(0, 1, 2, 3))]
    for r in reqs:
        assert serve.estimate_bytes(r, False, 150e9) < 150e9, r.kind
    assert serve.rixs_streamed(reqs[2], 150e9)
    small = Request("rixs", ModelSpec(6, 8, 1), ngs=1, omegas=np.linspace(0, 8, 8), eloss=eloss, pols=(0,))
    assert not serve.rixs_streamed(small, 150e9)
