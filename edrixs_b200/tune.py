"""Autotuner for the launch shape of the fused SpMM + Lanczos-step kernel.

For a given resident matrix and column count it runs a few Lanczos steps per candidate
shape (columns per lane group, threads per block, blocks per SM, interleaved or chunked
row mapping), times the apply launches with the CUDA events libedx records on the launch
stream, times the four fastest again over twice the steps, and keeps the fastest of those.  Results are cached per (matrix, columns, precision).
"""
import torch

from . import device
from ._lib import EdxError

_cache = {}


def candidates(k):
    if k > 32:
        kws = [32, 16]
    else:
        # the smallest group width >= k, and the next power of two (fewer idle lanes vs
        # simpler slot reduction)
        widths = [1, 2, 4, 6, 8, 12, 16, 32]
        first = next(w for w in widths if w >= k)
        pow2 = next(w for w in (1, 2, 4, 8, 16, 32) if w >= k)
        kws = sorted({first, pow2})
    shapes = [(256, 4), (256, 8), (1024, 1), (1024, 2)]
    out = []
    for kw in kws:
        tiles = [1]
        if kw >= 16:
            nt = (k + kw - 1) // kw
            tiles = [t for t in (1, 2, 4) if t <= nt]
        for tg in tiles:
            for th, bps in shapes:
                for ch in (0, 1):
                    out.append(dict(col_group=kw, tiles=tg, threads=th, blocks_per_sm=bps, chunked=ch))
    return out


def kron_candidates(k):
    """Launches of the slab product worth timing for k columns: staged source slabs, and
    source rows gathered from global memory on the default grid (32 blocks per SM, best for
    tens of millions of rows) and on 4 blocks per SM (best near a million rows)."""
    return [dict(col_group=device.KRON_STAGED), dict(col_group=device.KRON_GATHER),
            dict(col_group=device.KRON_GATHER, threads=256, blocks_per_sm=4)]


def tune_apply(A: device.CSR, k, c64=False, steps=3, verbose=False, packed=None, kron=None):
    """Fastest launch shape for k columns on A.  With a packed form or a slab form of A
    (complex128 only) their products are timed too; the result then carries "packed": 1 or
    "kron": 1."""
    key = (A.row_ptr.data_ptr(), A.nnz, k, bool(c64), packed is not None, kron is not None)
    if key in _cache:
        return _cache[key]
    dev = A.row_ptr.device
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    V0 = torch.randn((A.nrows, k), dtype=torch.float64, device=dev, generator=g).to(torch.complex128)
    results = []
    cands = candidates(k)
    if k <= 16:  # one row per lane group on the CSR too
        cands += [dict(c, rowslot=1) for c in candidates(k) if c["chunked"] == 0]
    if isinstance(A, device.PackedMatrix):  # no CSR: the packed product in every shape
        packed, cands = A, []
    if packed is not None and not c64:
        cands = cands + [dict(c, packed=1, rowslot=0) for c in candidates(k)]
        if k <= 16:  # one row per lane group
            cands += [dict(c, packed=1, rowslot=1) for c in candidates(k) if c["chunked"] == 0]
    if kron is not None and not c64:
        cands = cands + [dict(c, kron=1) for c in kron_candidates(k)]

    def args_of(cfg):
        if cfg.get("kron"):
            return dict({x: v for x, v in cfg.items() if x != "kron"}, kron=kron)
        if cfg.get("packed"):
            return dict(cfg, packed=packed)
        return cfg

    def time_of(cfg, nsteps):
        r = device.krylov(A, V0, nsteps, c64=c64, timing=True, apply=args_of(cfg))
        return r.apply_ms / max(r.apply_launches, 1)

    for cfg in cands:
        # one untimed step first: the first launch of a kernel also loads it
        try:
            device.krylov(A, V0, 1, c64=c64, apply=args_of(cfg))
        except EdxError:
            if cfg.get("kron"):  # a slab product variant this matrix does not fit (large slabs)
                continue
            raise
        results.append((time_of(cfg, steps), cfg))
    # the closest few again, and the fastest shape of each form (CSR, packed, slab), over more
    # steps, so that noise in the short first round (clocks move under the power cap) neither
    # picks the shape nor drops a form before the comparison
    results.sort(key=lambda x: x[0])

    def form(cfg):
        return "kron" if cfg.get("kron") else ("packed" if cfg.get("packed") else "csr")

    again = [cfg for _, cfg in results[:4]]
    for f in ("csr", "packed", "kron"):
        first = next((cfg for _, cfg in results if form(cfg) == f), None)
        if first is not None and first not in again:
            again.append(first)
    final = [(time_of(cfg, 3 * steps), cfg) for cfg in again]
    best_t, best = min(final, key=lambda x: x[0])
    # within 3% of the fastest, prefer the form that reads fewer matrix bytes (slab, then
    # packed, then CSR), then the smaller grid: such near-ties flip with noise, and the leaner
    # form shares HBM better
    lean = {"kron": 0, "packed": 1}
    near = [(t, c) for t, c in final if t <= 1.03 * best_t]
    best_t, best = min(near, key=lambda x: (min([lean[f] for f in lean if x[1].get(f)] + [2]),
                                            x[1].get("blocks_per_sm", 0), x[0]))
    del V0
    if verbose:
        for t, cfg in sorted(results, key=lambda x: x[0]):
            print(f"  {t * 1e3:9.1f} us  {cfg}")
    _cache[key] = dict(best, ms_per_launch=best_t)
    return _cache[key]
