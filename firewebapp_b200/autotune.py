"""The batched form's autotuner: picks the DOM sweep's cluster shape for a
number of cases stepped together on one GPU.

A single case's default sweep (path 8) takes 8 octant clusters of 10 CTAs, 80
of the 148 SMs, one CTA per SM; two cases' sweeps then cannot be resident at
once and mostly run one after the other.  Smaller clusters (6 CTAs per octant:
48 SMs, 22 such clusters resident) let two or three cases sweep at the same
time at some cost per sweep.  Which wins depends on the cases, the concurrency
and the form, so ``tune_batch`` times every candidate on the cases themselves
(``batch.time_concurrent``: fresh solvers, warm-up steps, then timed steps of
all cases at once) and keeps the fastest.  Results are cached in a JSON file
keyed by device, form, concurrency and the cases' grids.  Every candidate
gives the same results (the sweep paths are bit-identical), so tuning only
changes speed.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import torch

# (sweep path, CTAs per octant): path 8 automatic (10 on the 400x120x60 grid), 8, 7, 6
CANDIDATES = ((8, 0), (8, 8), (8, 7), (8, 6))


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
