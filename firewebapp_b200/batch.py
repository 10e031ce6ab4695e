"""Several independent Tier-3 cases stepped at once on one GPU (the batched form).

The reference runs one case per process (``run_3d_spread``); a parameter
sweep is many such runs.  Here ``run_batch`` keeps ``concurrency`` cases in
flight on one GPU, each with its own CUDA streams and host thread, and hands
the next case to whichever worker finishes first.  A single case leaves the
GPU partly idle (its DOM sweep holds 80 SMs while the rest wait for it, and
its host-side decisions - the adaptive dt, the pressure and DOM convergence
tests - pause its stream), so a second case's kernels fill those gaps.
Cases never exchange data and every kernel of a case is the one the single
-case solver launches, in the same order on the same stream, so each case's
result is bit-identical to running it alone.

Multi-GPU: the cases shard over ranks (``shard``) with no data-path
collective, as independent replicas.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import torch

from .solver import Tier3Solver


@dataclass
class BatchCaseResult:
    index: int
    cells: int
    steps: int
    t: float
    finished: str | None
    wall_s: float
    front_t: list = field(default_factory=list)
    front_x: list = field(default_factory=list)
    state: dict | None = None


def shard(n_cases: int, rank: int, world: int, weights=None) -> list[int]:
    """Case indices for ``rank`` of ``world``: greedy longest-first on
    ``weights`` (default: equal), so the ranks' total work is balanced."""
    w = list(weights) if weights is not None else [1.0] * n_cases
    order = sorted(range(n_cases), key=lambda i: -w[i])
    load = [0.0] * world
    own = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        own[r].append(i)
        load[r] += w[i]
    return sorted(own[rank])


def run_batch(cases, steps: int, form: str = "plain", concurrency: int = 2,
              device="cuda", keep_state: bool = False, warmup: int = 0,
              on_case_done=None, solver_kw: dict | None = None) -> list[BatchCaseResult]:
    """Step every case of ``cases`` for ``steps`` outer steps (fewer if the
    case ends, as the reference loop ends), ``concurrency`` cases at a time.
    ``warmup`` untimed steps precede the timed ones of each case.  Returns one
    ``BatchCaseResult`` per case, in input order; ``keep_state`` adds the
    final state (``Tier3Solver.state()``) to each.  ``solver_kw`` goes to every
    ``Tier3Solver`` (e.g. an ``autotune.tune_batch`` choice)."""
    if concurrency < 1:
        raise ValueError("concurrency must be >= 1")
    dev = torch.device(device)
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    results: list[BatchCaseResult | None] = [None] * len(cases)
    lock = threading.Lock()
    nxt = [0]
    errors: list[BaseException] = []

    def worker():
        try:
            torch.cuda.set_device(dev)
            stream = torch.cuda.Stream(device=dev)
            with torch.cuda.stream(stream):
                while True:
                    with lock:
                        if errors or nxt[0] >= len(cases):
                            return
                        i = nxt[0]
                        nxt[0] += 1
                    s = Tier3Solver(cases[i], device=dev, form=form, **(solver_kw or {}))
                    try:
                        for _ in range(warmup):
                            if not s.step():
                                break
                        stream.synchronize()
                        t0 = time.perf_counter()
                        n = 0
                        for _ in range(steps):
                            if not s.step():
                                break
                            n += 1
                        stream.synchronize()
                        wall = time.perf_counter() - t0
                        r = BatchCaseResult(index=i, cells=s.n, steps=n, t=s.t,
                                            finished=s.finished, wall_s=wall,
                                            front_t=list(s.front_t), front_x=list(s.front_x),
                                            state=s.state() if keep_state else None)
                    finally:
                        s.close()
                    results[i] = r
                    if on_case_done is not None:
                        on_case_done(r)
        except BaseException as e:  # surfaced to the caller below
            with lock:
                errors.append(e)

    threads = [threading.Thread(target=worker, name=f"case-worker-{w}")
               for w in range(min(concurrency, len(cases)))]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    return results


def time_concurrent(cases, steps: int, warmup: int = 3, form: str = "plain",
                    device="cuda", solver_kw: dict | None = None) -> dict:
    """Aggregate cell-steps/s of all ``cases`` stepped at the same time, one
    host thread and stream per case: every solver is built and warmed up
    first, then the timed region runs ``steps`` steps of every case between
    two device-wide synchronisations (host clock)."""
    dev = torch.device(device)
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    solvers, streams = [], []
    try:
        for c in cases:
            st = torch.cuda.Stream(device=dev)
            with torch.cuda.stream(st):
                s = Tier3Solver(c, device=dev, form=form, **(solver_kw or {}))
                for _ in range(warmup):
                    s.step()
            solvers.append(s)
            streams.append(st)
        torch.cuda.synchronize(dev)
        done = [0] * len(solvers)
        errors: list[BaseException] = []
        go = threading.Barrier(len(solvers) + 1, timeout=600)

        def run(q):
            try:
                torch.cuda.set_device(dev)
                with torch.cuda.stream(streams[q]):
                    go.wait()
                    for _ in range(steps):
                        if not solvers[q].step():
                            break
                        done[q] += 1
            except BaseException as e:
                errors.append(e)

        threads = [threading.Thread(target=run, args=(q,)) for q in range(len(solvers))]
        for th in threads:
            th.start()
        go.wait()
        t0 = time.perf_counter()
        for th in threads:
            th.join()
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        if errors:
            raise errors[0]
        work = sum(s.n * d for s, d in zip(solvers, done))
        return {"value": work / wall, "wall_s": wall, "cell_steps": work,
                "cells": [s.n for s in solvers], "steps": done}
    finally:
        for s in solvers:
            s.close()
