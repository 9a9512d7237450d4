"""Autotuner of the tiled H.v plan.

The tiled kernels (single-vector and R-vector) take three main plan
parameters: how many low global bits the tile rows keep (runs of consecutive
states, for coalescing), how many outer bits a pass expects to find in L2, and
at most how many passes the flip masks are split into.  The single-vector
kernel also takes the rows per thread (2^j_bits: 2048-state tiles at 3,
4096-state tiles at 4) and the resident blocks per SM.  Which combination is fastest
depends on the lattice, the vector count and the device, so the tuner times
the H.V of the actual model over a small candidate set and keeps the
fastest.  Results are cached in-process per (lattice, terms, R, device), and
optionally in a JSON file.
"""
from __future__ import annotations

import json
import os

from . import api

# (row_fixed_bits, window_bits, max_passes[, j_bits[, l1_carveout, stage_partner_tiles, blocks_per_sm[, objective[,
#  terms_in_flight]]]]);
# -1 = the library default.  Three resident blocks per SM pay up to about 2^26 states,
# 16-row tiles (j_bits 4) about 2^28.
CANDIDATES_1 = [(8, 10, 4, 3), (8, 8, 2, 3), (8, 10, 1, 3), (5, 8, 1, 3), (5, 10, 2, 3), (5, 12, 2, 3),
                (5, 12, 3, 3), (6, 12, 2, 3), (4, 12, 2, 3), (5, 14, 2, 3),
                (5, 12, 2, 2), (5, 10, 2, 2), (8, 10, 2, 2), (5, 13, 2, 2), (5, 12, 1, 2),
                (5, 12, 2, 1), (5, 10, 2, 1), (8, 10, 2, 1), (5, 13, 2, 1),
                (8, 8, 2, 3, 1, 0, 3), (5, 10, 2, 3, 1, 0, 3), (5, 11, 2, 3, 1, 0, 3), (8, 10, 4, 3, 1, 0, 3),
                (5, 11, 2, 4), (5, 10, 2, 4), (4, 11, 2, 4),
                # objective 1: tiles that hold the most flip terms
                (5, 10, 2, 3, 1, 0, -1, 1), (5, 8, 2, 3, 1, 0, -1, 1), (5, 10, 2, 4, 1, 0, -1, 1),
                (5, 9, 2, 4, 1, 0, -1, 1), (5, 11, 2, 4, 1, 0, -1, 1), (5, 10, 2, 3, 1, 0, 3, 1),
                (8, 8, 2, 3, 1, 0, -1, 1), (5, 10, 3, 4, 1, 0, -1, 1),
                # own rows, epilogue rows and diagonal by tensor copies (plans whose tiles
                # fit the copy geometry; the others are skipped)
                (5, 8, 2, 3, 1, 3, -1, 1), (5, 7, 2, 3, 1, 3, -1, 1), (5, 9, 2, 3, 1, 3, -1, 1),
                (5, 10, 2, 3, 1, 3, -1, 1), (5, 6, 2, 3, 1, 3, -1, 1), (5, 4, 2, 3, 1, 3, -1, 1),
                (5, 12, 2, 3, 1, 3, -1, 1), (5, 8, 3, 3, 1, 3, -1, 1),
                # the same with the partner rows of two out-of-tile terms in flight
                (5, 8, 2, 3, 1, 3, -1, 1, 2), (5, 7, 2, 3, 1, 3, -1, 1, 2), (5, 9, 2, 3, 1, 3, -1, 1, 2),
                (5, 10, 2, 3, 1, 3, -1, 1, 2), (5, 6, 2, 3, 1, 3, -1, 1, 2), (5, 4, 2, 3, 1, 3, -1, 1, 2),
                (5, 12, 2, 3, 1, 3, -1, 1, 2)]
CANDIDATES_R = [(-1, -1, -1), (0, 6, 2), (0, 8, 2), (0, 10, 2), (1, 10, 2), (3, 10, 2), (0, 10, 1),
                # objective 1: tiles on the bits that hold the most flip terms (rows need no low
                # bits: a state's R values are already a contiguous run)
                (0, 6, 2, -1, 1, 0, -1, 1), (0, 8, 2, -1, 1, 0, -1, 1), (0, 10, 2, -1, 1, 0, -1, 1),
                (1, 8, 2, -1, 1, 0, -1, 1), (0, 8, 3, -1, 1, 0, -1, 1), (0, 12, 1, -1, 1, 0, -1, 1)]

_cache: dict = {}


def _device_name():
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def _key(model, R):
    d = model.desc
    return f"n{d.n}-q{d.q}-b{d.n_bonds}-t{model.n_terms}-ip{hash(d._ipair.tobytes()) & 0xffffffff:08x}-R{R}"


def _time_hv(ctx, v1, v0, reps):
    import torch
    ctx.p_mltply_v3(v1, v0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        ctx.p_mltply_v3(v1, v0)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(model, R: int = 1, reps: int = 2, candidates=None, cache_path: str | None = None) -> dict:
    """Sets the fastest tile plan of `model` for R vectors; returns
    {"plan": (fixed, window, passes), "ms": H.V time, "tried": [...]}."""
    import torch
    key = f"{_key(model, R)}-{_device_name()}"
    if key not in _cache and cache_path and os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                _cache.update(json.load(f))
        except (OSError, ValueError):
            pass
    if key in _cache:
        best = _cache[key]
        model.set_plan(R, *best["plan"])
        return dict(best, cached=True)
    cands = candidates or (CANDIDATES_1 if R == 1 else CANDIDATES_R)
    ctx = api.Context(model, R=R)
    v1 = torch.randn(model.dim * R, dtype=torch.complex128, device="cuda")
    v0 = torch.zeros_like(v1)
    tried = []
    for c in cands:
        plan = model.set_plan(R, *c)
        if R == 1 and plan["tile_passes"] == 0:
            break                      # no tiled kernel for this model: nothing to tune
        if R == 1 and len(c) > 5 and c[5] == 3 and plan.get("staging") != 3:
            continue                   # tiles outside the tensor-copy geometry: the plan fell back
        tried.append({"plan": list(c), "ms": _time_hv(ctx, v1, v0, reps), "partner_tiles": plan["partner_tiles"],
                      "passes": plan["tile_passes"]})
    del v1, v0
    ctx.close()
    torch.cuda.empty_cache()
    if not tried:
        model.set_plan(R)
        return {"plan": [-1, -1, -1], "ms": None, "tried": []}
    best = min(tried, key=lambda t: t["ms"])
    model.set_plan(R, *best["plan"])
    _cache[key] = {"plan": best["plan"], "ms": best["ms"]}
    if cache_path:
        try:
            with open(cache_path, "w") as f:
                json.dump(_cache, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return {"plan": best["plan"], "ms": best["ms"], "tried": tried, "cached": False}


def autotune_slots(batch, structure, reps: int = 3, candidates=None) -> dict:
    """Sets the fastest tile plan of a slot batch: every slot runs a Lanczos
    chain of the (generic) structure couplings while each candidate plan is
    timed over `reps` batch steps; the slots are released afterwards."""
    import torch
    key = f"slots-n{structure.n}-b{structure.n_bonds}-R{batch.R}-{_device_name()}"
    if key in _cache:
        batch.set_plan(*_cache[key]["plan"])
        return dict(_cache[key], cached=True)
    if batch.plan()["tile_passes"] == 0:
        return {"plan": [-1, -1, -1], "ms": None, "tried": []}
    cands = candidates or (CANDIDATES_1 if batch.R == 1 else CANDIDATES_R)
    need = (reps + 1) * len(cands) + 2
    if need > batch.max_steps:
        cands = cands[:max(1, batch.max_steps // (reps + 1) - 1)]
    v = torch.empty(batch.dim, dtype=torch.complex128, device="cuda")
    stream = getattr(batch, "_stream", None)
    for r in range(batch.R):
        api.gaussian_column(batch.dim, batch.R, r, 12345, v)
        torch.cuda.synchronize()
        batch.load(r, "lanczos", structure, v, batch.max_steps)
    tried = []
    for c in cands:
        batch.set_plan(*c)
        batch.step(1)
        batch.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s = stream if stream is not None else torch.cuda.current_stream()
        e0.record(s)
        batch.step(reps)
        e1.record(s)
        batch.synchronize()
        torch.cuda.synchronize()
        tried.append({"plan": list(c), "ms": e0.elapsed_time(e1) / reps})
    for r in range(batch.R):
        batch.release(r)
    batch.synchronize()
    best = min(tried, key=lambda t: t["ms"])
    batch.set_plan(*best["plan"])
    _cache[key] = {"plan": best["plan"], "ms": best["ms"]}
    return {"plan": best["plan"], "ms": best["ms"], "tried": tried, "cached": False}
