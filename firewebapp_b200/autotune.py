"""The batched form's autotuner: picks the DOM sweep's shape for a number of
cases stepped together on one GPU.

A single case's default sweep (path 8) takes 8 octant clusters of 10 CTAs, 80
of the 148 SMs, one CTA per SM, so two cases' sweeps cannot be resident at
once.  The other shapes trade differently: 6-CTA clusters take two clusters
per octant (an S8 octant's intensities for 10 rows of 120 pencils do not fit
one CTA's shared memory), 16 clusters on 96 SMs; 15-CTA clusters run in two
waves on 120 SMs.  Which is fastest next to the other cases' kernels depends
on the cases, the concurrency and the form, so ``tune_batch`` times every
candidate on the cases themselves (``batch.time_concurrent``: fresh solvers,
warm-up steps, then timed steps of all cases at once) and keeps the fastest.
Results are cached in a JSON file keyed by device, form, concurrency and the
cases' grids.  The shapes agree to rounding (about 1e-15 relative in the
radiative sources; the two-cluster shape also sums each octant's G in two
halves).
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import torch

# (sweep path, CTAs per octant): path 8 automatic (10 CTAs per octant on the
# 60 x 120 cross-section), 6-CTA clusters (two per octant), 15-CTA clusters
CANDIDATES = ((8, 0), (8, 6), (8, 15))


def cache_path() -> Path:
    return Path(os.environ.get("FIREWEBAPP_B200_TUNE_CACHE",
                               Path.home() / ".cache" / "firewebapp_b200" / "tune.json"))


def cache_key(cases, concurrency: int, form: str, device_name: str) -> str:
    from .grid import build_setup
    shapes = sorted({tuple(build_setup(c).grid.shape) for c in cases})
    return (f"{device_name}|{form}|conc{concurrency}|"
            + ";".join("x".join(map(str, s)) for s in shapes))


def tune_batch(cases, concurrency: int = 2, form: str = "plain", steps: int = 4,
               warmup: int = 3, candidates=CANDIDATES, device="cuda", use_cache: bool = True,
               log=None) -> dict:
    """Best ``Tier3Solver`` keyword arguments (``dom_sweep``,
    ``dom_cluster_ctas``) for stepping ``concurrency`` of ``cases`` at once,
    timed on the first ``concurrency`` cases.  Returns {"solver_kw": ...,
    "trials": [{"solver_kw", "value", "wall_s"}, ...], "cached": bool}."""
    from .batch import time_concurrent
    from ._lib import FireStepError
    sample = list(cases[:max(1, concurrency)])
    key = cache_key(sample, concurrency, form, torch.cuda.get_device_name(device))
    path = cache_path()
    cache = {}
    if path.exists():
        try:
            cache = json.loads(path.read_text())
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        out = dict(cache[key])
        out["cached"] = True
        return out
    trials = []
    for mode, ctas in candidates:
        kw = {"dom_sweep": mode, "dom_cluster_ctas": ctas}
        try:
            r = time_concurrent(sample, steps, warmup=warmup, form=form, device=device,
                                solver_kw=kw)
        except FireStepError as e:  # a cluster shape this grid cannot take
            trials.append({"solver_kw": kw, "value": 0.0, "error": str(e)})
            continue
        trials.append({"solver_kw": kw, "value": r["value"], "wall_s": r["wall_s"]})
        if log:
            log(f"autotune {key}: {kw} -> {r['value']:.3e} cell-steps/s")
    best = max(trials, key=lambda t: t["value"])
    if not best["value"] > 0.0:
        raise RuntimeError(f"autotune {key}: no candidate ran")
    out = {"key": key, "solver_kw": best["solver_kw"], "trials": trials}
    cache[key] = out
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(cache, indent=1))
    except OSError:
        pass
    out = dict(out)
    out["cached"] = False
    return out
