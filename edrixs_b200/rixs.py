"""Batched RIXS on one resident problem: every incident energy, polarisation pair and ground
state of a request in one pass.

The reference (edrixs/solvers.py:2651-2702 -> src/rixs_driver.f90) loops over incident
energies omega, polarisation pairs and ground states g; each iteration rebuilds H_n, runs
MINRES (src/linsys.f90) on (omega + E_g + i*Gamma_c - H_n) x = D_in|g>, applies D_out^+,
rebuilds H_f and runs a 150-step Lanczos (src/lanczos.f90:210-303) for the poles.

Here:
 1. the seeds D_in(pol_in)|g> are one SpMM;
 2. the Lanczos vectors of H_n are the same for every shift z = omega + E_g + i*Gamma_c of
    one seed (src/linsys.f90 only ever uses alpha = <v, A v> = z - <v, H v>), so all
    incident energies of a seed share ONE Krylov space: k = (#pol_in x #gs) columns, one
    SpMM per iteration, with each shift's MINRES recurrence carried in that basis
    (libedx edx_krylov shifts) and stopped by the reference's own rule;
 3. every Lanczos vector is pushed through each D_out^+(pol_out) while it is hot in L2
    (edx_krylov projections), so x_z never has to exist: D_out^+ x_z = (D_out^+ V) y_z is
    a batched ZGEMM.  When the projected vectors would not fit in memory (``stream``), a
    second Krylov pass regenerates the same Lanczos vectors (deterministic reductions) and
    folds each D_out^+ v_i into the final-state start vectors, a window of
    ``stream_window`` steps at a time (edx_krylov proj_window);
 4. all #pol_out x #pol_in x #gs x #omega final-state Lanczos runs on H_f go as one block
    of columns (one SpMM per step);
 5. continued fractions for every pole set on the energy-loss grid (edx_cf_spectrum) and
    the Boltzmann sum over ground states (edrixs/utils.py:54-73).
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import device

KB = 8.6173303e-5


def boltz(gs_e, T):
    gs_e = np.asarray(gs_e, dtype=np.float64)
    w = np.exp(-(gs_e - gs_e.min()) / (KB * T))
    return w / w.sum()


@dataclass
class RixsProblem:
    """Resident device state of one RIXS Hamiltonian (what the server keeps in HBM)."""
    Hn: device.CSR
    Hf: device.CSR
    Din: List[device.CSR]
    Dout: List[device.CSR]
    gs_e: np.ndarray
    gs_v: torch.Tensor                       # (n_i, ngs) complex128
    meta: dict = field(default_factory=dict)
    packed: dict = field(default_factory=dict)  # "hf" / "hn" -> device.PackedMatrix of that matrix
    kron: dict = field(default_factory=dict)    # "hf" / "hn" -> device.KronMatrix (slab form) of that matrix

    def nbytes(self):
        b = self.Hn.nbytes() + self.Hf.nbytes() + sum(D.nbytes() for D in self.Din + self.Dout)
        if getattr(self.Hn, "val64", None) is not None:
            b += self.Hn.nnz * 8
        b += sum(M.nbytes() for M in self.packed.values())
        b += sum(M.nbytes() for M in self.kron.values())
        return b + self.gs_v.numel() * 16

    def dout_on_slabs(self):
        """D_out with its columns in the slab order of H_n (for projecting Lanczos vectors that
        live in that order); built once and kept."""
        key = ("dout_slab", id(self.kron["hn"]))
        if key not in self.meta:
            inv = self.kron["hn"].inv
            self.meta[key] = [device.relabel_columns(D, inv) for D in self.Dout]
        return self.meta[key]


def _apply_args(cfg, packed, c64, kron=None):
    """Launch arguments of one Krylov call: the autotuner's choice, else the packed product
    when a packed form exists (measured faster than the slab product on both matrices of the
    batched workload), else the slab product when only a slab form exists (a resident that
    keeps no per-entry matrix), else libedx's defaults."""
    if cfg is not None:
        if cfg.get("kron"):
            if kron is None:
                raise ValueError("the tuned launch shape needs the slab form")
            return dict({x: v for x, v in cfg.items() if x in ("col_group", "threads", "blocks_per_sm")}, kron=kron)
        if cfg.get("packed"):
            if packed is None:
                raise ValueError("the tuned launch shape needs the packed form")
            return dict(cfg, packed=packed)
        return cfg
    if packed is not None and not c64:
        return dict(packed=packed)
    if kron is not None and not c64:
        return dict(kron=kron)
    return None


@dataclass
class RixsResult:
    spectra: np.ndarray      # (n_omega, n_eloss, n_pol_in * n_pol_out), ordered (pol_in, pol_out)
    poles: dict              # alpha, beta (K, nkryl), norm, neff, e0 per final-state Lanczos run
    iters: np.ndarray        # MINRES iterations per (pol_in, gs, omega)
    res: np.ndarray          # |res| estimates
    krylov_steps: int        # Lanczos steps taken on H_n
    stats: dict = field(default_factory=dict)  # kernel launch counts and timings
    spectra_gs: Optional[np.ndarray] = None  # per ground state, before the Boltzmann sum:
    #                                          (n_omega, n_eloss, n_pol_in * n_pol_out, ngs)
    start: Optional[torch.Tensor] = None     # (n_f, len(start_cols)) final-state start vectors
    #                                          D_out^+ x of the requested columns


def _stream_needed(P, k, maxn):
    """True when storing D_out^+ v_i for every Lanczos vector would take more than a third of
    the free device memory (then the two-pass streaming form is used)."""
    free, _ = torch.cuda.mem_get_info()
    stored = sum(D.nrows for D in P.Dout) * k * maxn * 16
    return stored > free / 3


def rixs_spectra(P: RixsProblem, omegas, gamma_c, eloss, gamma_f, *, nkryl=150, linsys_tol=1e-10,
                 linsys_max=1000, temperature=300.0, c64=False, final_block=None, timing=False, autotune=False,
                 stream=None, stream_window=8, seeds=None, c64_final=None, per_gs=False, start_cols=None):
    """RIXS spectra of every (omega_in, pol_in, pol_out, gs) of one request.
    stream: None (automatic), True or False -- whether D_out^+ v_i is folded into the
    final-state start vectors as the Lanczos vectors appear (two passes over H_n) instead of
    being stored for every v_i.  seeds: the block D_in(pol_in)|g> (n_n, npin * ngs), column
    p_in * ngs + g, when the caller computed it already (P.Din is then not used).  c64: the
    H_n products (MINRES part) in complex64; c64_final: the H_f products too (default: as c64).
    per_gs: also return the spectra of each ground state before the Boltzmann sum.
    start_cols: final-state columns (p_out, p_in, g, omega order: column
    ((p_out * n_pol_in + p_in) * ngs + g) * n_omega + w) whose start vectors D_out^+ x to
    return in ``start``."""
    c64_f = c64 if c64_final is None else bool(c64_final)
    omegas = np.asarray(omegas, dtype=np.float64)
    eloss = np.asarray(eloss, dtype=np.float64)
    n_om, ne = len(omegas), len(eloss)
    npout, ngs = len(P.Dout), len(P.gs_e)
    npin = len(P.Din) if seeds is None else seeds.shape[1] // ngs
    k_hn = npin * ngs
    K_hf = npout * k_hn * n_om if final_block is None else int(final_block)
    if autotune:
        from . import tune
        P.meta[("apply", "hn", k_hn, c64)] = tune.tune_apply(P.Hn, k_hn, c64=c64, packed=P.packed.get("hn"),
                                                             kron=P.kron.get("hn"))
        P.meta[("apply", "hf", K_hf, c64_f)] = tune.tune_apply(P.Hf, K_hf, c64=c64_f, packed=P.packed.get("hf"),
                                                               kron=P.kron.get("hf"))
    cfg_hn = _apply_args(P.meta.get(("apply", "hn", k_hn, c64)), P.packed.get("hn"), c64, P.kron.get("hn"))
    cfg_hf = _apply_args(P.meta.get(("apply", "hf", K_hf, c64_f)), P.packed.get("hf"), c64_f, P.kron.get("hf"))
    # on the slab form of H_n the Lanczos vectors are in its slab order: seeds go in permuted,
    # and D_out^+ reads them through columns relabelled to that order
    Kn = cfg_hn.get("kron") if cfg_hn else None
    Kf = cfg_hf.get("kron") if cfg_hf else None
    dout = P.dout_on_slabs() if Kn is not None else P.Dout
    gam_c = np.broadcast_to(np.asarray(gamma_c, dtype=np.float64), (n_om,))
    dev = P.gs_v.device
    # 1. seeds (n_n, npin*ngs), column c = p_in*ngs + g
    if seeds is None:
        seeds = torch.cat([device.spmm(D, P.gs_v) for D in P.Din], dim=1).contiguous()
    k = seeds.shape[1]
    seeds_k = Kn.to_slab(seeds) if Kn is not None else seeds
    # 2. shifts: for every column its n_om incident energies
    scol = np.repeat(np.arange(k, dtype=np.int32), n_om)
    gsE = np.tile(P.gs_e, npin)
    sz = (omegas[None, :] + gsE[:, None] + 1j * gam_c[None, :]).reshape(-1)
    maxn = int(linsys_max)
    if stream is None:
        stream = _stream_needed(P, k, maxn)
    nf = P.Dout[0].nrows
    K = npout * k * n_om
    # 3. one Krylov space per seed + projections through every D_out^+
    if not stream:
        r = device.krylov(P.Hn, seeds_k, maxn, c64=c64, proj=dout, shifts=(scol, sz), shift_tol=linsys_tol,
                          shift_maxit=linsys_max, timing=timing, apply=cfg_hn)
    else:  # pass 1: the shifted recurrences alone
        r = device.krylov(P.Hn, seeds_k, maxn, c64=c64, shifts=(scol, sz), shift_tol=linsys_tol,
                          shift_maxit=linsys_max, timing=timing, apply=cfg_hn)
    steps = int(r.neff.max().item())
    m = max(int(r.shift_iters.max().item()), 1)
    iters = r.shift_iters.view(k, n_om).cpu().numpy()
    resid = r.shift_res.view(k, n_om).cpu().numpy()
    it_n = r.apply_launches
    # libedx launches on H_n: 4 setup + the first projections, then per iteration apply, orth,
    # shift step and per emission operator a projection and its column scaling
    stats = dict(hn_iterations=it_n, hn_apply_ms=r.apply_ms, hn_nnz=P.Hn.nnz, hn_rows=P.Hn.nrows, k_hn=k,
                 launches=npin + 4 + npout + it_n * (3 + 2 * npout) + (Kn is not None) + (Kf is not None),
                 streamed=bool(stream))
    if not stream:
        # V0[:, (p_out * k + c) * n_om + w] = sum_{i < m} Y[c, w, i] * (D_out(p_out)^+ v_i)[c]
        V0 = device.proj_combine(r.proj, r.shift_y, k, n_om, m)   # (n_f, K) row-major
        stats["launches"] += npout * k
        del r
    else:
        # pass 2: the same m Lanczos vectors again (deterministic reductions: the same
        # vectors), each D_out^+ v_i folded into phi as it appears, B vectors at a time
        Y = r.shift_y[:, :m].contiguous()                          # (k * n_om, m)
        r1_ms = r.apply_ms
        del r
        V0 = torch.zeros((nf, K), dtype=torch.complex128, device=dev)
        nacc = k * n_om
        outs = [V0[:, po * nacc:(po + 1) * nacc] for po in range(npout)]
        r2 = device.krylov(P.Hn, seeds_k, m, c64=c64, proj=dout, timing=timing, apply=cfg_hn,
                           accumulate=dict(window=int(stream_window), col=scol, coef=Y, out=outs))
        stats["hn_iterations"] += r2.apply_launches
        if timing:
            stats["hn_apply_ms"] = (r1_ms or 0.0) + (r2.apply_ms or 0.0)
        stats["launches"] += 4 + npout + r2.apply_launches * (2 + 2 * npout) + \
            npout * ((m + int(stream_window) - 1) // int(stream_window))
        del r2, Y
    start = V0[:, list(start_cols)].clone() if start_cols is not None else None
    if Kf is not None:  # the final-state Lanczos runs in the slab order of H_f
        V0 = Kf.to_slab(V0)
    # 4. final-state Lanczos, all pole sets as one block (optionally in chunks of columns)
    blk = K if final_block is None else int(final_block)
    A = torch.zeros((K, nkryl), dtype=torch.float64, device=dev)
    B = torch.zeros_like(A)
    NRM = torch.zeros(K, dtype=torch.float64, device=dev)
    NEFF = torch.zeros(K, dtype=torch.int32, device=dev)
    hf_ms, hf_it = 0.0, 0
    for s in range(0, K, blk):
        e = min(K, s + blk)
        rf = device.krylov(P.Hf, V0[:, s:e], nkryl, c64=c64_f, timing=timing, apply=cfg_hf)
        A[s:e], B[s:e], NRM[s:e], NEFF[s:e] = rf.alpha, rf.beta, rf.norm, rf.neff
        hf_ms += rf.apply_ms or 0.0
        hf_it += rf.apply_launches
        stats["launches"] += 2 + 2 * rf.apply_launches  # norm, start; apply + orth per step
    stats.update(hf_apply_ms=hf_ms if timing else None, hf_iterations=hf_it, hf_nnz=P.Hf.nnz, hf_rows=P.Hf.nrows,
                 k_hf=blk,
                 hf_packed=bool(cfg_hf and cfg_hf.get("packed") is not None),
                 hn_packed=bool(cfg_hn and cfg_hn.get("packed") is not None),
                 hf_kron=Kf is not None, hn_kron=Kn is not None)
    del V0
    # 5. continued fractions; column order (p_out, p_in, g, w)
    e0 = np.tile(np.repeat(np.tile(P.gs_e, npin), n_om), npout)
    spec = device.cf_spectrum(NEFF, A, B, e0, NRM.cpu().numpy(), np.ones(K), eloss,
                              np.broadcast_to(np.asarray(gamma_f, dtype=np.float64), (ne,)), per_set=True)
    spec = spec.view(npout, npin, ngs, n_om, ne)
    w = torch.from_numpy(boltz(P.gs_e, temperature)).to(dev)
    out = torch.einsum("oigwe,g->weio", spec, w).reshape(n_om, ne, npin * npout)
    stats["launches"] += 1
    per_g = spec.permute(3, 4, 1, 0, 2).reshape(n_om, ne, npin * npout, ngs).cpu().numpy() if per_gs else None
    return RixsResult(out.cpu().numpy(), dict(alpha=A, beta=B, norm=NRM, neff=NEFF, e0=e0), iters, resid, steps,
                      stats, per_g, start)


def rixs_request(P: RixsProblem, gs_v_host, omegas, gamma_c, eloss, gamma_f, **kw):
    """A request as a client makes it: ground-state vectors and grids in host memory,
    spectra back in host memory.  The vectors are copied from pinned host buffers into the
    resident problem before the solve."""
    P.gs_v.copy_(gs_v_host, non_blocking=True)
    return rixs_spectra(P, omegas, gamma_c, eloss, gamma_f, **kw)


def rixs_plain(P: RixsProblem, omega, gamma_c, eloss, gamma_f, *, pin=0, pout=0, g=0, nkryl=150, linsys_tol=1e-10,
               linsys_max=1000):
    """The reference's algorithm for ONE (omega, pol pair, ground state): one-RHS FP64 MINRES
    on H_n, D_out^+ x, one-column Lanczos on H_f.  Returns (alpha, beta, norm, neff, iters)."""
    b = device.spmm(P.Din[pin], P.gs_v[:, g].contiguous())
    z = complex(omega + P.gs_e[g], gamma_c)
    x, it, res = device.minres(P.Hn, b, linsys_tol, linsys_max, alpha=-1.0, sigma=z)
    phi = device.spmm(P.Dout[pout], x)
    rf = device.krylov(P.Hf, phi.reshape(-1, 1), nkryl)
    return rf, it, res
