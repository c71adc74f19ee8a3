"""Phase tracing for the solvers.

The reference prints the CPU time of its phases (src/ed_driver.f90:54,114-121,175-181,271-278)
and progress every 50 Krylov / MINRES iterations.  Here a phase is a ``with
trace.phase(name):`` block.  With the environment variable EDX_TRACE set to 1 (or
``trace.enable()``), each phase

* opens an NVTX range of its name, so that Nsight tools show the solver's phases over the
  kernels they launch;
* records a CUDA event on the current stream at either end and, when the phase closes, its
  device time next to its wall time in ``trace.records``;
* prints one line per phase when EDX_TRACE=2.

Disabled (the default), a phase costs one flag test and adds no synchronisation.
"""
import contextlib
import os
import time

_level = int(os.environ.get("EDX_TRACE", "0") or 0)
records = []


def enable(level=1):
    global _level
    _level = int(level)


def enabled():
    return _level > 0


@contextlib.contextmanager
def phase(name):
    if _level <= 0:
        yield
        return
    import torch
    cuda = torch.cuda.is_available()
    ev0 = ev1 = None
    if cuda:
        torch.cuda.nvtx.range_push(name)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
    t0 = time.perf_counter()
    ok = False
    try:
        yield
        ok = True
    finally:
        dev_ms = None
        if cuda:
            ev1.record()
            ev1.synchronize()
            dev_ms = ev0.elapsed_time(ev1)
            torch.cuda.nvtx.range_pop()
        rec = {"phase": name, "wall_ms": (time.perf_counter() - t0) * 1e3, "device_ms": dev_ms, "ok": ok}
        records.append(rec)
        if _level >= 2:
            dev = "" if dev_ms is None else f", device {dev_ms:.3f} ms"
            print(f"edx >>> {name}: wall {rec['wall_ms']:.3f} ms{dev}", flush=True)


def summary():
    """Total wall and device milliseconds per phase name over ``records``."""
    out = {}
    for r in records:
        s = out.setdefault(r["phase"], {"calls": 0, "wall_ms": 0.0, "device_ms": 0.0})
        s["calls"] += 1
        s["wall_ms"] += r["wall_ms"]
        if r["device_ms"] is not None:
            s["device_ms"] += r["device_ms"]
    return out
