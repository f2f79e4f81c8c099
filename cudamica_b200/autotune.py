"""Measured choice of the fused E-step's tile shape and launch shape.

The fused mixed-form E-step (up to 128 channels) is compiled in three tile
shapes (amica_cfg.tc_shape): 0 = 3 density warpgroups and 48-sample tiles with
2 TMA stages of x, 1 = 2 warpgroups and 32-sample tiles with 2 stages, 2 = 2
warpgroups with 3 stages.  The shape sets the samples per tile (MMA1 N, MMA2
K), the density warps per SM and the x pipeline depth; the fastest depends on
n (lane packing), M (cluster size) and m (registers and tensor-memory
columns for the log2|y| cache), so best_tile_shape times each on the
context's own data (the reference derives its launch shapes from n and the
SM count instead, src/helpers.cu:55-511).

The kernels are persistent: one cluster of M CTAs (one CTA per SM) per stream
of sample tiles, as many clusters as fit by default.  Also tunable is how many
clusters a context runs -- alone on the GPU the fastest grid, inside a cohort
of contexts that run concurrently the split of the SMs between subjects (or
none: every subject on the whole GPU, their streams interleaving).  All are
chosen from measurements (amica_time_estep for one context, timed cohort
iterations for a cohort); results are cached per problem shape for the
process, and optionally in a JSON file.
"""
from __future__ import annotations

import json
import os
from typing import Iterable, Sequence

from .engine import Amica

_cache: dict = {}


def _key(eng: Amica) -> str:
    return f"{eng.n}:{eng.T}:{eng.M}:{eng.m}:{eng.kernel}"


def load_cache(path: str) -> None:
    if os.path.exists(path):
        _cache.update(json.load(open(path)))


def save_cache(path: str) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(_cache, f, indent=1, sort_keys=True)


def estep_profile(eng: Amica, grids: Iterable[int], reps: int = 5) -> dict:
    """E-step ms at each grid cap (clusters; 0 = all that fit), measured on
    the context's own data and parameters.  Leaves the grid at the full size."""
    out = {}
    for g in grids:
        real = eng.set_grid(g)
        ms, _ = eng.time_estep(reps)
        out[real] = ms
    eng.set_grid(0)
    return out


TILE_SHAPES = (0, 1, 2)


def tile_shape_profile(eng: Amica, reps: int = 5) -> dict:
    """E-step ms of the context in each tile shape on its own data and
    parameters (full grid).  Leaves the context in shape 0."""
    out = {}
    for sh in TILE_SHAPES:
        eng.set_tile_shape(sh)
        eng.estep_stats()                     # first launch of this shape, untimed
        out[sh] = eng.time_estep(reps)[0]
    eng.set_tile_shape(0)
    return out


def best_tile_shape(eng: Amica, reps: int = 5) -> int:
    """The fastest tile shape for the context's (n, T, M, m), measured once
    per problem shape and cached; the context is left in it.  Contexts that
    do not run the fused form keep their kernel (returns -1)."""
    if eng.kernel != "tc_tf32":
        return -1
    key = "tile:" + _key(eng)
    if key not in _cache:
        prof = tile_shape_profile(eng, reps)
        _cache[key] = {"best": min(prof, key=prof.get), "ms": {str(k): v for k, v in prof.items()}}
    best = int(_cache[key]["best"])
    eng.set_tile_shape(best)
    return best


def best_grid(eng: Amica, tolerance: float = 0.03, reps: int = 5) -> int:
    """The smallest grid whose E-step time is within `tolerance` of the fastest
    measured (full grid, 3/4, 1/2, 1/4 of it): alone on the GPU, fewer clusters
    at equal speed leave SMs free for other streams."""
    key = "best:" + _key(eng)
    if key in _cache:
        return int(_cache[key])
    full = eng.set_grid(0)
    cands = sorted({full, max(1, (3 * full) // 4), max(1, full // 2), max(1, full // 4)})
    prof = estep_profile(eng, cands, reps)
    fastest = min(prof.values())
    pick = min(g for g, ms in prof.items() if ms <= fastest * (1.0 + tolerance))
    _cache[key] = pick
    return pick


def split_budget(work: Sequence[float], budget: int, weights: Sequence[int] = None) -> list:
    """Clusters per subject for subjects sharing `budget` SMs concurrently,
    each cluster occupying weights[s] SMs (its model count M): proportional to
    the measured work (ms of E-step on the full GPU), at least one cluster each,
    largest remainders first.  Pure host logic."""
    S = len(work)
    if S == 0:
        return []
    weights = list(weights) if weights is not None else [1] * S
    total = float(sum(work)) or 1.0
    # SMs each subject should get, then clusters
    ideal = [budget * w / total for w in work]
    alloc = [max(1, int(ideal[s] // weights[s])) for s in range(S)]
    used = sum(alloc[s] * weights[s] for s in range(S))
    order = sorted(range(S), key=lambda s: ideal[s] - alloc[s] * weights[s], reverse=True)
    for s in order:
        if used + weights[s] <= budget and ideal[s] - alloc[s] * weights[s] > 0:
            alloc[s] += 1
            used += weights[s]
    return alloc


def cohort_grids(engines: Sequence[Amica], sm_budget: int, reps: int = 3) -> list:
    """Grid caps for contexts that will run concurrently: each subject's E-step
    is timed on the whole GPU, then the SMs are split in proportion."""
    work = []
    for eng in engines:
        key = "full:" + _key(eng)
        if key not in _cache:
            eng.set_grid(0)
            _cache[key] = eng.time_estep(reps)[0]
        work.append(float(_cache[key]))
    return split_budget(work, sm_budget, [eng.M for eng in engines])


def tune_cohort(engines: Sequence[Amica], sm_budget: int, reset, iters: int = 4,
                budgets: Sequence[float] = (1.0, 0.8)) -> tuple[list, dict]:
    """Pick the grids of a cohort by timing real cohort iterations under each
    candidate: every subject on the whole GPU (grid 0), or the SMs split in
    proportion to the subjects' work at each fraction of `sm_budget`.  `reset()`
    restores the subjects' starting state afterwards.  Returns (grids, ms per
    cohort iteration for each candidate)."""
    import time
    key = "cohort:" + ",".join(_key(e) for e in engines) + f":{sm_budget}"
    if key in _cache:
        grids = list(_cache[key]["grids"])
        return grids, dict(_cache[key]["timings"])
    cands = {"whole_gpu": [0] * len(engines)}
    work = cohort_grids(engines, sm_budget)   # measures and caches the work
    work_ms = [float(_cache["full:" + _key(e)]) for e in engines]
    for f in budgets:
        cands[f"split_{f:g}"] = split_budget(work_ms, max(len(engines), int(sm_budget * f)),
                                             [e.M for e in engines])
    del work
    timings = {}
    for name, grids in cands.items():
        for e, g in zip(engines, grids):
            e.set_grid(g)
        for e in engines:
            e.run_async(1)
        for e in engines:
            e.run_wait()
        t0 = time.perf_counter()
        for e in engines:
            e.run_async(iters)
        for e in engines:
            e.run_wait()
        timings[name] = (time.perf_counter() - t0) * 1e3 / iters
    reset()
    best = min(timings, key=timings.get)
    grids = cands[best]
    for e, g in zip(engines, grids):
        e.set_grid(g)
    _cache[key] = {"grids": grids, "timings": timings, "choice": best}
    return list(grids), timings
