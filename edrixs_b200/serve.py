"""Continuous-batching request loop for ED / XAS / RIXS jobs on one GPU.

* Requests name a Hamiltonian by its generating parameters (``ModelSpec``); the server keeps
  each Hamiltonian's product form, transition operators and ground states resident in HBM
  (``Resident``) and reuses them for later requests.  The product form is the packed matrix
  (its CSR is dropped once packed), or, for intermediate sectors above SLAB_ONLY_ROWS rows,
  the slab form alone: no CSR is built at all (at 58 M rows the CSR takes 114 GB while it is
  packed, the packed form 35 GB, the slab form 0.9 GB, and the slab product runs the
  few-column recurrences as fast as the packed one).
* Admission: a request starts when its estimated device footprint (its resident problem if
  not cached yet + its solve working set) fits in the HBM budget next to everything in
  flight; idle residents are evicted least-recently-used to make room.  Requests that do
  not fit wait; requests larger than the whole budget fail at admission.
* Coalescing: waiting RIXS requests on the same Hamiltonian with the same broadening and
  solver settings are merged into one multi-shift solve over the union of their incident
  energies (their shifts share Krylov spaces), then split back per request.
* Continuous batching: several worker threads, each with its own CUDA stream, run admitted
  work concurrently; a request that arrives while others run is admitted as soon as memory
  and a worker free up.  Every request records its queueing and service latency.
* Cancellation: a caller may cancel a request's Future while the request waits; it then
  leaves the queue (and any coalesced solve).  Once its solve starts it can no longer be
  cancelled (concurrent.futures semantics).
"""
import itertools
import math
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import device, rixs, siam, solvers

KB = 8.6173303e-5


@dataclass(frozen=True)
class ModelSpec:
    """A seeded SIAM Hamiltonian: 10 impurity + nbath bath valence orbitals, 2p core."""
    nbath: int
    nelec: int
    seed: int

    @property
    def nv(self):
        return 10 + self.nbath


@dataclass
class Request:
    kind: str                      # "ed", "xas" or "rixs"
    model: ModelSpec
    ngs: int = 1                   # ground states used (lowest ngs)
    omegas: Optional[np.ndarray] = None   # rixs: incident energies relative to the edge
    eloss: Optional[np.ndarray] = None    # rixs: energy-loss grid; xas: absorption grid
    gamma_c: float = 0.6
    gamma_f: float = 0.1
    pols: tuple = (0,)             # rixs: indices into siam.rixs_polarisations(); xas: xas polvec index
    nkryl: int = 150
    linsys_tol: float = 1e-10
    linsys_max: int = 1000
    temperature: float = 300.0
    id: int = field(default_factory=lambda: next(_ids))
    t_submit: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0


_ids = itertools.count()


# intermediate sectors above this many rows are held in the slab form alone (when the model
# has one): no CSR is built, and at 57.9 M rows its product is faster than the packed one
# (57-61 against 66-68 ms for 6 columns).  Below it the packed form, whose product is as fast
# as the slab form's on its default grid at 1 M rows (0.72 against 0.70 ms)
SLAB_ONLY_ROWS = 20_000_000
# rows below which the CSR itself is kept (the eigensolver's dense path needs it)
SMALL_ROWS = 4096
# bytes per row, for the admission estimate: a complex128 CSR while it is built and packed
# (up to ~100 entries per row at 26 orbitals), its packed form, the slab form (row
# permutation, its inverse and tables) and the transient of building the slab form
CSR_ROW, PACKED_ROW, SLAB_ROW, SLAB_BUILD_ROW = 2048 + 640, 640, 24, 64
# basis vectors of the ground-state eigensolver (block thick-restart Lanczos)
ED_BASIS = 64
# final-state Lanczos columns per launch in the server (bounds its working set)
FINAL_BLOCK = 64
# Lanczos vectors folded at a time into the final-state start vectors (streamed RIXS)
STREAM_WINDOW = 4


def _product_form(mode, basis, hop, coul, nv, nc, slab_first):
    """The matrix a resident keeps for products: the slab form when slab_first and the model
    has one (no CSR is built), else the packed form with its CSR dropped, else (too many
    distinct values, or a small matrix) the CSR."""
    if slab_first:
        K = device.kron_form(mode, basis, hop, coul, num_val_orbs=nv, num_core_orbs=nc)
        if K is not None:
            return K
    H = device.build_csr(mode, basis, hop, coul, num_val_orbs=nv, num_core_orbs=nc)
    if H.nrows < SMALL_ROWS:
        return H
    P = device.pack(H)
    return P if P is not None else H


class Resident:
    """Device state of one Hamiltonian, built on first use.  Hi / Hn: the product form of
    H_i and H_n (device.PackedMatrix, device.KronMatrix or device.CSR, see _product_form)."""

    def __init__(self, spec: ModelSpec):
        self.spec = spec
        self.lock = threading.Lock()
        self.Hi = None
        self.Hn = None
        self.bi = self.bn = None
        self.terms = None
        self.model = None
        self.gs_e = None
        self.gs_v = None
        self.edge = None
        self.ops = {}
        self.busy = 0
        self.last_used = time.monotonic()

    def nbytes(self):
        b = 0
        for M in [self.Hi, self.Hn] + list(self.ops.values()):
            if M is not None:
                b += M.nbytes()
        if self.gs_v is not None:
            b += self.gs_v.numel() * 16
        return b

    def ensure(self, need_n=False, ngs=1):
        """Build what is missing and return a snapshot (gs_e, gs_v) of the ground states.
        A later request for more ground states replaces gs_e and gs_v; a solve uses only its
        own snapshot, so it never mixes the eigenvalues of one set with the vectors of another."""
        with self.lock:
            s = self.spec
            if self.model is None:
                self.model = siam.make_siam(s.nbath, s.nelec, s.seed)
                m, rt = self.model, siam.text_roundtrip
                self.terms = dict(hop_i=rt(siam.nonzero_terms(m.emat_i), 2), coul_i=rt(siam.nonzero_terms(m.umat_i), 4),
                                  hop_n=rt(siam.nonzero_terms(m.emat_n), 2), coul_n=rt(siam.nonzero_terms(m.umat_n), 4))
            if self.Hi is None:
                self.bi = device.fock_unrank(s.nv, s.nelec)
                self.Hi = _product_form(device.HAM_I, self.bi, self.terms["hop_i"], self.terms["coul_i"], s.nv, 0,
                                        slab_first=False)
            if self.gs_v is None or self.gs_v.shape[1] < ngs:
                # two guard vectors in the block: a level just above the wanted ones (a
                # near-degenerate pair across the boundary) otherwise stalls their residuals
                e, v = solvers.lowest_eigs(self.Hi, ngs, ngs, tol=1e-9, block=min(ngs + 2, 6), mmax=ED_BASIS)
                self.gs_e, self.gs_v = np.asarray(e), v.contiguous()
            if need_n and self.Hn is None:
                self.bn = device.fock_unrank(s.nv, s.nelec + 1)
                nn = 6 * self.bn.ndim
                self.Hn = _product_form(device.HAM_N, self.bn, self.terms["hop_n"], self.terms["coul_n"], s.nv, 6,
                                        slab_first=nn > SLAB_ONLY_ROWS)
                if isinstance(self.Hn, device.KronMatrix):
                    # the absorption edge from a plain Lanczos run (a few vectors, not the
                    # block eigensolver's basis of tens of GB at this size)
                    e_n, _ = solvers.plain_lanczos_eigs(self.Hn, 1, 0, 400, 1e-9)
                else:
                    e_n, _ = solvers.lowest_eigs(self.Hn, 1, 1, tol=1e-6)
                self.edge = float(e_n[0] - self.gs_e[0])
            # the resident is shared with other workers' streams: finish building it here
            torch.cuda.current_stream().synchronize()
            self.last_used = time.monotonic()
            return self.gs_e, self.gs_v

    def op(self, kind, pol):
        key = (kind, pol)
        with self.lock:
            if key not in self.ops:
                m, rt, s = self.model, siam.text_roundtrip, self.spec
                pols = siam.rixs_polarisations()
                if kind == "in":
                    t = rt(siam.nonzero_terms(siam.polarised_operator(m, pols[pol][0])), 2)
                    self.ops[key] = device.build_csr(device.TRANS_I, self.bn, t, right=self.bi, num_val_orbs=s.nv,
                                                     num_core_orbs=6)
                elif kind == "out":
                    t = rt(siam.nonzero_terms(np.conj(siam.polarised_operator(m, pols[pol][1])).T), 2)
                    self.ops[key] = device.build_csr(device.TRANS_F, self.bi, t, right=self.bn, num_val_orbs=s.nv,
                                                     num_core_orbs=6)
                else:  # xas
                    t = rt(siam.nonzero_terms(siam.polarised_operator(m, siam.atomic()["xas_polvec"][pol])), 2)
                    self.ops[key] = device.build_csr(device.TRANS_I, self.bn, t, right=self.bi, num_val_orbs=s.nv,
                                                     num_core_orbs=6)
                torch.cuda.current_stream().synchronize()
            return self.ops[key]


def _dims(spec: ModelSpec):
    ni = math.comb(spec.nv, spec.nelec)
    nn = 6 * math.comb(spec.nv, spec.nelec + 1)
    return ni, nn


def _rixs_shape(req: Request):
    """(k, npout, K): Lanczos columns on H_n (incident polarisations x ground states),
    outgoing polarisations, final-state columns."""
    npin = len(set(siam_pol_in(p) for p in req.pols))
    npout = len(set(siam_pol_out(p) for p in req.pols))
    k = npin * req.ngs
    return k, npout, npout * k * len(req.omegas)


def rixs_streamed(req: Request, budget):
    """Whether the server runs this RIXS request in the streamed form (D_out^+ v_i folded into
    the final-state start vectors as the Lanczos vectors appear) rather than storing every
    projected vector: when storing them would take more than a quarter of the HBM budget."""
    ni, _ = _dims(req.model)
    k, npout, _ = _rixs_shape(req)
    return npout * k * req.linsys_max * ni * 16 > budget / 4


def estimate_bytes(req: Request, resident_cached: bool, budget=150e9):
    """Upper estimate of the device bytes a request needs: its resident problem when not
    cached yet (the product forms it keeps, plus the larger of the build transients: a CSR
    while it is packed, or the slab form's row tables, and the edge's eigensolver basis) and
    the working set of its solve."""
    ni, nn = _dims(req.model)
    resident = 0
    if not resident_cached:
        keep = ni * PACKED_ROW
        peak = ni * CSR_ROW + (ED_BASIS + 8) * ni * 16  # build of H_i, then the ground-state basis
        if req.kind != "ed":
            if nn > SLAB_ONLY_ROWS:
                keep += nn * SLAB_ROW
                peak = max(peak, nn * SLAB_BUILD_ROW, 6 * nn * 16)
            else:
                keep += nn * PACKED_ROW
                peak = max(peak, nn * CSR_ROW, 48 * nn * 16)
        resident = keep + peak
    if req.kind == "ed":
        work = 2 * (ED_BASIS + 8) * ni * 16
    elif req.kind == "xas":
        work = 6 * nn * 16 * max(req.ngs, 1)
    else:
        k, npout, K = _rixs_shape(req)
        ops = (npout * ni * 30 + 2 * nn * 5) * 20  # D_out (and a relabelled copy), D_in
        hn_phase = 6 * nn * k + K * ni
        if rixs_streamed(req, budget):
            hn_phase += STREAM_WINDOW * npout * k * ni
        else:
            hn_phase += npout * k * req.linsys_max * ni
        final_phase = K * ni + 4 * ni * min(K, FINAL_BLOCK)
        work = ops + max(hn_phase, final_phase) * 16
    return int(resident + work)


def coalesce_key(req: Request):
    """Requests with equal keys share one solve: RIXS on one Hamiltonian with the same
    linewidths, Lanczos and MINRES settings, temperature and loss grid (their incident
    energies, polarisations and ground-state counts may differ: the solve takes the union and
    the largest count, and each request gets its own columns and Boltzmann sum back); XAS on
    one Hamiltonian with the same Lanczos length (one Krylov launch over all their start
    vectors).  ED requests are not coalesced."""
    if req.kind == "rixs":
        return ("rixs", req.model, req.gamma_c, req.gamma_f, req.nkryl, req.linsys_tol, req.linsys_max,
                req.temperature, len(req.eloss), float(req.eloss[0]), float(req.eloss[-1]))
    if req.kind == "xas":
        return ("xas", req.model, req.nkryl)
    return None


class Server:
    def __init__(self, hbm_budget=150e9, workers=2):
        self.budget = float(hbm_budget)
        self.workers = workers
        self.residents = {}
        self.waiting = []            # [(req, future)]
        self.inflight_bytes = 0
        self.cv = threading.Condition()
        self.jobs = queue.Queue()
        self.stop_flag = False
        self.records = []
        self.threads = []
        # a request is taken from the waiting list only when a worker is free, so that the
        # requests which arrive meanwhile can join its solve (coalesce_key)
        self.free_workers = workers

    # -- public ---------------------------------------------------------------------------
    def start(self):
        device.require_cuda()
        _warm_torch()
        self.sched = threading.Thread(target=self._schedule, daemon=True)
        self.sched.start()
        for i in range(self.workers):
            t = threading.Thread(target=self._work, args=(i,), daemon=True)
            t.start()
            self.threads.append(t)
        return self

    def submit(self, req: Request) -> Future:
        fut = Future()
        req.t_submit = time.perf_counter()
        if estimate_bytes(req, False, self.budget) > self.budget:
            fut.set_exception(MemoryError(f"request {req.id} needs more than the HBM budget"))
            return fut
        with self.cv:
            if self.stop_flag:
                fut.set_exception(RuntimeError(f"request {req.id}: the server is shut down"))
                return fut
            self.waiting.append((req, fut))
            self.cv.notify_all()
        return fut

    def shutdown(self):
        """Stop taking work.  Requests still waiting are cancelled (their futures raise
        CancelledError); solves already running finish first."""
        with self.cv:
            self.stop_flag = True
            for _, fut in self.waiting:
                fut.cancel()
            self.waiting = []
            self.cv.notify_all()
        for _ in self.threads:
            self.jobs.put(None)
        for t in self.threads:
            t.join(timeout=60)

    def latency_summary(self):
        lat = np.array([r["latency_s"] for r in self.records]) if self.records else np.zeros(1)
        return {"n": len(self.records), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3)}

    # -- scheduling -----------------------------------------------------------------------
    def _resident(self, spec):
        if spec not in self.residents:
            self.residents[spec] = Resident(spec)
        return self.residents[spec]

    def _resident_bytes(self):
        return sum(r.nbytes() for r in self.residents.values())

    def _evict_for(self, need):
        idle = sorted((r for r in self.residents.values() if r.busy == 0), key=lambda r: r.last_used)
        for r in idle:
            if self._resident_bytes() + self.inflight_bytes + need <= self.budget:
                break
            del self.residents[r.spec]

    def _schedule(self):
        while True:
            with self.cv:
                if self.stop_flag:
                    return
                # requests whose callers cancelled them (Future.cancel) leave the queue
                self.waiting = [(r, f) for r, f in self.waiting if not f.cancelled()]
                if self.free_workers == 0 or not self.waiting:
                    self.cv.wait(timeout=0.05)
                    continue
                picked = None
                for i, (req, fut) in enumerate(self.waiting):
                    cached = req.model in self.residents
                    need = estimate_bytes(req, cached, self.budget)
                    if self._resident_bytes() + self.inflight_bytes + need > self.budget:
                        self._evict_for(need)
                    if self._resident_bytes() + self.inflight_bytes + need <= self.budget:
                        picked = i
                        break
                if picked is None:
                    self.cv.wait(timeout=0.05)
                    continue
                req, fut = self.waiting.pop(picked)
                group = [(req, fut)]
                sig = coalesce_key(req)
                if sig is not None:  # waiting requests that can share this one's solve
                    rest = []
                    for r2, f2 in self.waiting:
                        (group if coalesce_key(r2) == sig else rest).append((r2, f2))
                    self.waiting = rest
                # a future marked running can no longer be cancelled; one cancelled since the
                # purge above is dropped here
                group = [(r, f) for r, f in group if f.set_running_or_notify_cancel()]
                if not group:
                    continue
                req = group[0][0]
                need = sum(estimate_bytes(r, r.model in self.residents, self.budget) for r, _ in group)
                res = self._resident(req.model)
                res.busy += 1
                self.inflight_bytes += need
                self.free_workers -= 1
                # queued while the lock is held: shutdown() takes the lock before it queues
                # the workers' stop markers, so a picked job always reaches a worker first
                self.jobs.put((group, res, need))

    def _work(self, idx):
        stream = torch.cuda.Stream()
        while True:
            job = self.jobs.get()
            if job is None:
                return
            group, res, need = job
            t0 = time.perf_counter()
            try:
                with torch.cuda.stream(stream):
                    outs = self._run(group, res)
                    stream.synchronize()
                t1 = time.perf_counter()
                for (req, fut), out in zip(group, outs):
                    req.t_start, req.t_done = t0, t1
                    self.records.append({"id": req.id, "kind": req.kind, "latency_s": t1 - req.t_submit,
                                         "service_s": t1 - t0, "coalesced": len(group),
                                         "norb": req.model.nv, "dims": _dims(req.model)})
                    fut.set_result(out)
            except Exception as e:  # a failed job fails its requests, never the server
                for req, fut in group:
                    if not fut.done():
                        fut.set_exception(e)
            finally:
                with self.cv:
                    res.busy -= 1
                    self.inflight_bytes -= need
                    self.free_workers += 1
                    self.cv.notify_all()

    # -- solves ---------------------------------------------------------------------------
    def _run(self, group, res: Resident):
        req = group[0][0]
        if req.kind == "ed":
            gs_e, _ = res.ensure(False, req.ngs)
            return [{"eigvals": gs_e[:r.ngs].copy()} for r, _ in group]
        G = max(r.ngs for r, _ in group)
        gs_e, gs_v = res.ensure(True, G)
        # this stream reads the snapshot: if another request replaces it meanwhile, the
        # caching allocator keeps its memory until the work queued here has finished
        gs_v.record_stream(torch.cuda.current_stream())
        if req.kind == "xas":
            return self._xas_group(group, res, gs_e, gs_v)
        # union of incident energies (absolute) and polarisations over the coalesced requests
        oms = [np.asarray(r.omegas, dtype=np.float64) + res.edge for r, _ in group]
        allw = np.unique(np.concatenate(oms))
        pins = sorted(set(siam_pol_in(p) for r, _ in group for p in r.pols))
        pouts = sorted(set(siam_pol_out(p) for r, _ in group for p in r.pols))
        forms = {}
        for key, M in (("hf", res.Hi), ("hn", res.Hn)):
            if isinstance(M, device.PackedMatrix):
                forms.setdefault("packed", {})[key] = M
            elif isinstance(M, device.KronMatrix):
                forms.setdefault("kron", {})[key] = M
        P = rixs.RixsProblem(Hn=res.Hn, Hf=res.Hi, Din=[res.op("in", p) for p in pins],
                             Dout=[res.op("out", p) for p in pouts], gs_e=gs_e[:G],
                             gs_v=gs_v[:, :G].contiguous(), **forms)
        widest = max((r for r, _ in group), key=lambda r: _rixs_shape(r)[0])
        out = rixs.rixs_spectra(P, allw, req.gamma_c, req.eloss, req.gamma_f, nkryl=req.nkryl,
                                linsys_tol=req.linsys_tol, linsys_max=req.linsys_max, temperature=req.temperature,
                                per_gs=True, stream=rixs_streamed(widest, self.budget), stream_window=STREAM_WINDOW,
                                final_block=FINAL_BLOCK)
        results = []
        for (r, _), om in zip(group, oms):
            idx = np.searchsorted(allw, om)
            cols = [pins.index(siam_pol_in(p)) * len(pouts) + pouts.index(siam_pol_out(p)) for p in r.pols]
            w = rixs.boltz(gs_e[:r.ngs], r.temperature)  # this request's own ground states
            spec = np.einsum("weng,g->wen", out.spectra_gs[idx][:, :, cols, :r.ngs], w)
            results.append({"omegas": om, "spectra": spec, "coalesced": len(group), "minres_iters": out.iters})
        return results

    def _xas_group(self, group, res: Resident, gs_e, gs_v):
        """XAS of every request in the group from one Krylov launch: the start vectors
        D_xas(pol)|g> of all of them side by side (build_krylov_mp per column, as the
        reference runs them one by one), then each request's continued fraction.  gs_e, gs_v:
        the ground-state snapshot this solve took."""
        phis, spans = [], []
        c0 = 0
        for r, _ in group:
            phis.append(device.spmm(res.op("xas", r.pols[0]), gs_v[:, :r.ngs].contiguous()))
            spans.append((c0, c0 + r.ngs))
            c0 += r.ngs
        phi = torch.cat(phis, dim=1).contiguous()
        if isinstance(res.Hn, device.KronMatrix):  # the slab product, on start vectors in its row order
            kr = device.krylov(res.Hn, res.Hn.to_slab(phi), group[0][0].nkryl)
        else:
            kr = device.krylov(res.Hn, phi, group[0][0].nkryl)
        norm = kr.norm.cpu().numpy()
        out = []
        for (r, _), (a, b) in zip(group, spans):
            w = rixs.boltz(gs_e[:r.ngs], r.temperature)
            grid = np.asarray(r.eloss, dtype=np.float64) + res.edge
            spec = device.cf_spectrum(kr.neff[a:b], kr.alpha[a:b], kr.beta[a:b], gs_e[:r.ngs], norm[a:b], w,
                                      grid, np.full(len(grid), r.gamma_c))
            out.append({"grid": grid, "spectrum": spec.cpu().numpy(), "coalesced": len(group)})
        return out


def _warm_torch():
    """Run once, on the calling thread, every torch routine the solves use: torch loads some
    of its linear-algebra backends lazily, and that first load must not happen in several
    worker threads at once."""
    A = torch.randn((8, 8), dtype=torch.complex128, device="cuda")
    H = A + A.conj().T
    torch.linalg.qr(A, mode="reduced")
    torch.linalg.eigh(H)
    torch.linalg.vector_norm(A, dim=0, keepdim=True)
    torch.matmul(A, A)
    torch.einsum("ij,j->i", A, A[0])
    torch.cuda.synchronize()


def siam_pol_in(p):
    """Incident polarisation of rixs_polarisations()[p]: entries 0,1 share pi, 2,3 share sigma."""
    return 0 if p in (0, 1) else 2


def siam_pol_out(p):
    """Outgoing polarisation of rixs_polarisations()[p]: entries 0,2 share pi, 1,3 share sigma."""
    return 0 if p in (0, 2) else 1
