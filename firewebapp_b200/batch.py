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

import numpy as np
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


def _print_line(text):
    print(text, flush=True)


def main(argv=None):
    """``python -m firewebapp_b200.batch --cases 32 --steps 2000 --concurrency 4``:
    the batched sweep of uneven domains (``cases.batch_cases``) through the
    work queue of ``run_batch``; one JSON line per case as it finishes, then a
    summary line (cell-steps/s over the whole sweep by the host clock)."""
    import argparse
    import json
    from .cases import batch_cases
    ap = argparse.ArgumentParser(description="batched sweep of independent Tier-3 cases")
    ap.add_argument("--cases", type=int, default=32)
    ap.add_argument("--seed0", type=int, default=0)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--concurrency", type=int, default=4)
    ap.add_argument("--form", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--engine", default="python", choices=["python", "ctx"],
                    help="python: Tier3Solver work queue (run_batch); ctx: groups of "
                         "--concurrency whole-step contexts stepped together from C++ "
                         "(fs_batch_run, no interpreter lock while stepping)")
    args = ap.parse_args(argv)
    cases = batch_cases(args.cases, seed0=args.seed0)
    if args.engine == "ctx":
        return _main_ctx(cases, args)

    out_lock = threading.Lock()

    def done(r):
        c = cases[r.index]
        with out_lock:
            _print_line(json.dumps({"case": r.index, "cells": r.cells, "nx": int(round(c["Lx"] / c["dx"])),
                          "U10": c["wind_speed_m_s"], "steps": r.steps, "t": r.t,
                          "finished": r.finished, "wall_s": r.wall_s,
                          "cell_steps_per_s": r.cells * r.steps / max(r.wall_s, 1e-12)}))

    t0 = time.perf_counter()
    res = run_batch(cases, args.steps, form=args.form, concurrency=args.concurrency,
                    on_case_done=done)
    wall = time.perf_counter() - t0
    work = sum(r.cells * r.steps for r in res)
    print(json.dumps({"cases": len(res), "steps_per_case": args.steps,
                      "concurrency": args.concurrency, "form": args.form,
                      "cell_steps": work, "wall_s": wall, "cell_steps_per_s": work / wall,
                      "note": "wall clock includes each case's set-up"}), flush=True)



def _main_ctx(cases, args):
    """The sweep through whole-step contexts: each group of ``concurrency``
    cases is built (host set-up), then stepped together by ``fs_batch_run``
    (one C++ host thread and stream pair per case)."""
    import json
    from .ctx import StepContext, batch_run
    t0 = time.perf_counter()
    work, step_wall = 0, 0.0
    for g0 in range(0, len(cases), args.concurrency):
        idx = list(range(g0, min(g0 + args.concurrency, len(cases))))
        ctxs = [StepContext(cases[i], form=args.form) for i in idx]
        try:
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            outs = batch_run(ctxs, args.steps)
            dt = time.perf_counter() - t1
            step_wall += dt
            cells = [int(np.prod(c.shape)) for c in ctxs]
            gw = sum(n * o.steps for n, o in zip(cells, outs))
            work += gw
            _print_line(json.dumps({"group": idx, "cells": cells,
                                    "steps": [o.steps for o in outs],
                                    "finished": [int(o.finished) for o in outs],
                                    "wall_s": dt, "cell_steps_per_s": gw / dt}))
        finally:
            for c in ctxs:
                c.close()
    wall = time.perf_counter() - t0
    _print_line(json.dumps({"cases": len(cases), "steps_per_case": args.steps,
                            "concurrency": args.concurrency, "form": args.form,
                            "engine": "ctx", "cell_steps": work, "wall_s": wall,
                            "cell_steps_per_s": work / wall,
                            "stepping_cell_steps_per_s": work / step_wall,
                            "note": "wall_s includes each group's set-up; the stepping "
                                    "figure times the fs_batch_run calls only"}))


if __name__ == "__main__":
    main()
