#!/usr/bin/env python
"""Benchmark of the Tier-3 step: 3D solver cell-steps/s on B200.

Workload: the 400 x 120 x 60 cell case (2.88M cells, dx = dy = 0.1 m,
dz = 0.0625 m, DOM S8 with 80 ordinates, U10 = 6 m/s, moisture 0.06,
rho_b = 0.35 kg/m^3, 16 bed particles per surface cell, seeded jitter), plain
FP64 path, projection tolerance 1e-6 (the reference's production default).
Synthetic initial state built from the case deck (no dataset exists for this
solver).  Inputs exceed L2 (state ~0.7 GB + DOM intensities 1.84 GB), so no
L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank advances its own
independent replica of the case ("replicas only": the single-case step does
not shard); value = cell-steps/s summed over ranks, time = max over ranks.
``--impl reference`` times the CPU restatement of the reference algorithm
(oracle/) on the host on a bounded slice of the same workload.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "3D solver cell-steps/s on 1 B200 (plain FP64 Tier-3 step)"
UNIT = "cell-steps/s"
WORKLOAD = "tier3_step_400x120x60_S8_fp64"
# measured DRAM bytes per cell of one launch (see the traffic comment in main)
TRAFFIC_PER_CELL = {"dom_sweep": (16.7488e6 + 3.00672e6) / 720000.0}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def job_totals(cells_steps: float, seconds: float, device="cpu"):
    """Whole-job work and time over the ranks: cell-steps summed, time the
    maximum (the slowest rank bounds the job).  Single process: unchanged."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(cells_steps), float(seconds)
    w = torch.tensor([float(cells_steps)], dtype=torch.float64, device=device)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(w.item()), float(t.item())


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """SM clocks and clock-event reasons sampled (NVML, read-only queries,
    every 50 ms) while the timed region runs."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, cuda_index):
        self.idx = cuda_index
        self.samples = []
        self._stop = threading.Event()
        self._th = None
        self.handle = None
        self.max_mhz = None
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(cuda_index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self.nv = nv
            self.handle = nv.nvmlDeviceGetHandleByUUID(uuid)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.handle, nv.NVML_CLOCK_SM))
        except Exception:
            self.handle = None

    def start(self):
        if self.handle is None:
            return

        def run():
            nv = self.nv
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                    self.samples.append((float(sm), int(rs)))
                except Exception:
                    pass
                self._stop.wait(0.05)
        self._th = threading.Thread(target=run, daemon=True)
        self._th.start()

    def stop(self):
        self._stop.set()
        if self._th:
            self._th.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(s for s, _ in self.samples),
                "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples), "source": "nvml"}


def _oracle_slice(case_nx, seed=0):
    """Oracle state for the workload restricted to its first ``case_nx`` x-cells."""
    from firewebapp_b200.cases import CFG2, scaled
    from firewebapp_b200.grid import build_setup
    from firewebapp_b200.quadrature import level_symmetric
    from oracle.step import OracleState, geometry_from_setup
    case = dict(scaled(CFG2, nx=case_nx), jitter_seed=seed)
    su = build_setup(case)
    snap = dict(su.fields)
    snap["T_soil"] = su.soil["T"]
    for k, v in su.particles.items():
        snap["p_" + k] = v
    om, wq = level_symmetric(8)
    S = OracleState(snap, geometry_from_setup(su), su.params, om, wq)
    S.proj_solver = "bicgstab"
    S.proj_rtol = 1.0e-6
    return S, su.grid.n_cells


def cpu_sample(nx_slice=50, steps=1):
    """Time the oracle port on a bounded slice (one or more outer steps)."""
    from oracle.step import step
    S, cells = _oracle_slice(nx_slice)
    t0 = time.perf_counter()
    for _ in range(steps):
        step(S)
    el = time.perf_counter() - t0
    return cells * steps / el, cells, el


def _ref_worker(nx_slice, warmup, steps, seed, q):
    """One host process: the oracle on its own slice replica (spawned)."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle.step import step
    S, cells = _oracle_slice(nx_slice, seed)
    for _ in range(warmup):
        step(S)
    q.put(("ready", seed))
    t0 = time.perf_counter()
    for _ in range(steps):
        step(S)
    q.put(("done", cells * steps, time.perf_counter() - t0))


def run_reference_arm(args):
    """The CPU restatement on the host cores: one spawned process per core
    (capped), each stepping its own replica of an x-slice of the workload."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    import multiprocessing as mp
    nx_slice = int(os.environ.get("FIRE_REF_SLICE_NX", "25"))
    try:
        ncpu = len(os.sched_getaffinity(0))
    except AttributeError:
        ncpu = os.cpu_count() or 1
    nproc = max(1, min(ncpu, int(os.environ.get("FIRE_REF_MAX_PROCS", "16"))))
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=(nx_slice, args.warmup, args.steps, r, q))
             for r in range(nproc)]
    for pr in procs:
        pr.start()
    work, times = 0, []
    for _ in range(2 * nproc):
        msg = q.get(timeout=3600)
        if msg[0] == "done":
            work += msg[1]
            times.append(msg[2])
    for pr in procs:
        pr.join()
    el = max(times)
    value = work / el
    cells = work // (nproc * args.steps)
    sample = (f"{nproc} processes x {args.steps} outer steps, each on its own replica of the "
              f"first {nx_slice} x-cells of the {WORKLOAD} case ({cells} cells), numpy "
              f"oracle port, projection BiCGSTAB rtol 1e-6, value = all work / slowest process")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"x-slice of {nx_slice} cells",
                   "parallelism": f"host x{nproc}"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batch_bench(args):
    """N cases of the batched sweep (``cases.batch_cases``) on each GPU: all
    stepped concurrently (one stream and host thread per case), and the same
    cases one after another; both aggregate cell-steps/s over the timed steps,
    host clock between device-wide synchronisations.  Ranks take disjoint
    cases (weak scaling, no collective on the data path)."""
    import torch
    import torch.distributed as dist
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    from firewebapp_b200.batch import time_concurrent
    from firewebapp_b200.cases import batch_cases
    cases = batch_cases(args.batch, seed0=rank * args.batch)
    tuned = None
    kw = {}
    if args.autotune:
        from firewebapp_b200.autotune import tune_batch
        tuned = tune_batch(cases, concurrency=len(cases), form=args.form, use_cache=False)
        kw = tuned["solver_kw"]
    conc = time_concurrent(cases, args.steps, warmup=args.warmup, form=args.form, solver_kw=kw)
    seq_work, seq_wall = 0.0, 0.0
    for c in cases:
        one = time_concurrent([c], args.steps, warmup=args.warmup, form=args.form)
        seq_work += one["cell_steps"]
        seq_wall += one["wall_s"]
    work, wall = conc["cell_steps"], conc["wall_s"]
    if ws > 1:
        t = torch.tensor([work, wall, seq_work, seq_wall], dtype=torch.float64, device="cuda")
        parts = [torch.zeros_like(t) for _ in range(ws)]
        dist.all_gather(parts, t)
        tot = torch.stack(parts)
        work, seq_work = float(tot[:, 0].sum()), float(tot[:, 2].sum())
        wall, seq_wall = float(tot[:, 1].max()), float(tot[:, 3].max())
    if rank == 0:
        line = {
            "metric": METRIC.replace("plain FP64 Tier-3 step", "batched sweep"), "value": work / wall,
            "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * wall / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.form == "plain" else "f64+f32", "data": "synthetic",
            "config": {"workload": f"tier3_batch_{args.batch}_cases_nx200-600_S8_{args.form}",
                       "cases_per_gpu": args.batch, "cells": conc["cells"],
                       "parallelism": f"replicas{ws}", "timing": "host clock between "
                       "device-wide synchronisations"},
            "sequential_value": seq_work / seq_wall,
            "concurrency_gain": (work / wall) / (seq_work / seq_wall),
            "autotune": ({"solver_kw": tuned["solver_kw"],
                          "trials": [{"solver_kw": t["solver_kw"], "value": t["value"]}
                                     for t in tuned["trials"]]} if tuned else None),
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--form", default="plain", choices=["plain", "mixed", "learned"],
                    help="plain: FP64 throughout; mixed: FP32 DOM sweep and multigrid "
                         "preconditioner, pressure tolerance 1e-8; learned: mixed with the "
                         "pressure solve in flexible CG preconditioned by the trained U-Net "
                         "(bf16 tensor-core convolutions), V-cycle fallback on a stall")
    ap.add_argument("--no-clocks", action="store_true",
                    help="skip the clock sampler (diagnostics only; the line then has no clocks)")
    ap.add_argument("--nx", type=int, default=None,
                    help="run the workload cut to its first NX x-cells (profiling)")
    ap.add_argument("--dom-sweep", type=int, default=0,
                    help="force a DOM sweep path (fs_dom_set_sweep_mode); 0 picks automatically")
    ap.add_argument("--batch", type=int, default=0,
                    help="instead of the headline line: N cases of the batched sweep of uneven "
                         "domains (Nx 200-600) stepped concurrently, against the same cases "
                         "stepped one after another")
    ap.add_argument("--autotune", action="store_true",
                    help="with --batch: pick the DOM cluster shape for the concurrent cases "
                         "by timing each candidate on them first (autotune.tune_batch)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.batch:
        run_batch_bench(args)
        return

    import torch
    import torch.distributed as dist
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    from firewebapp_b200 import _lib
    from firewebapp_b200.cases import CFG2
    from firewebapp_b200.solver import Tier3Solver

    case = dict(CFG2, jitter_seed=rank)
    if args.nx:
        from firewebapp_b200.cases import scaled
        case = dict(scaled(CFG2, nx=args.nx), jitter_seed=rank)
    solver = Tier3Solver(case, form=args.form, dom_sweep=args.dom_sweep)
    cells = solver.n
    for _ in range(args.warmup):
        solver.step()
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            dist.barrier()

    # ---- timed region: device-resident state, CUDA events on the stream
    # Objects alive now (torch, numpy, the solver) move to the permanent GC
    # generation, so a full collection during the steps scans only new ones.
    gc.collect()
    gc.freeze()
    solver.enable_kernel_timers(True)
    lib = _lib.lib()
    clocks = ClockSampler(local) if not args.no_clocks else None
    if clocks:
        clocks.start()
    barrier()
    torch.cuda.synchronize()
    n0 = lib.fs_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        solver.step()
    e1.record()
    torch.cuda.synchronize()
    launches = int(lib.fs_launch_count() - n0)
    barrier()
    clk = clocks.stop() if clocks else {"sm_mhz": None, "reasons": ["not sampled"]}
    ms = e0.elapsed_time(e1) / args.steps
    kt = solver.kernel_times()
    solver.enable_kernel_timers(False)
    work, sec = job_totals(cells * args.steps, ms * 1e-3 * args.steps, device="cuda")
    ms = 1e3 * sec / args.steps
    value = work / sec

    # ---- roofline of the dominant bracketed kernel
    peak, peak_src = _peaks()
    N = cells
    M = solver.Omega.shape[0]
    dom_mode = lib.fs_dom_sweep_mode(solver.dom)
    alg = {  # algorithmic bytes per launch (distinct fields read + written, 8 B each)
        # octant sweeps (paths 1, 4, 6, 7, 8): read (kappa, kappa*B) once and write
        # the 8 octant partial G fields (FP32 in the mixed form; wrap rows and
        # ground partials < 1% more); per-ordinate paths write every intensity
        "dom_sweep": (N * (8.0 + 4.0 * 8) if args.form != "plain" else
                      N * (16.0 + 8.0 * 8) if dom_mode in (1, 4, 6, 7, 8) else N * (8.0 * M + 16.0)),
        "species_transport": N * 8.0 * 12,
        "edc": N * 8.0 * 11,
        "turb_diffusion_Y": N * 8.0 * 7,
        "momentum_drag": N * 8.0 * 10,
        "k_epsilon": N * 8.0 * 14,
        "gas_energy_adv": N * 8.0 * 5,
    }
    dom_k = max((k for k in kt if k in alg), key=lambda k: kt[k][0])
    tot_ms, nl = kt[dom_k]
    avg_ms = tot_ms / max(nl, 1)
    achieved = alg[dom_k] / (avg_ms * 1e-3) / 1e9
    # DRAM bytes per launch of the dominant kernel from an ncu capture of the
    # 100x120x60 slice of this workload (dram__bytes_read.sum + write.sum) with
    # the default sweep (path 8), scaled by the cell count to a full launch
    traffic = (TRAFFIC_PER_CELL.get(dom_k)
               if args.form == "plain" and (dom_k != "dom_sweep" or dom_mode == 8) else None)
    if traffic is not None:
        traffic *= N
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": dom_k,
                "peak_source": peak_src, "launches": nl, "avg_launch_ms": avg_ms,
                "algorithmic_bytes_per_launch": alg[dom_k], "dom_sweep_path": dom_mode,
                "kernels_ms_per_step": {k: v[0] / args.steps for k, v in kt.items()}}

    # ---- end to end through the public API: host state in, result out
    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(case, args.steps, ws, args.form)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, c, el = cpu_sample(nx_slice=50, steps=1)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"1 outer step of the {WORKLOAD} case on its first 50 x-cells "
                         f"({c} cells, {el:.1f} s), numpy oracle port, projection "
                         f"BiCGSTAB rtol 1e-6"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"plain": "f64", "mixed": "f64+f32"}.get(args.form, "f64+f32+bf16"),
            "data": "synthetic",
            "config": {"workload": (WORKLOAD if not args.nx else
                                    f"tier3_step_{args.nx}x120x60_S8_fp64").replace(
                                        "fp64", "fp64" if args.form == "plain" else args.form),
                       "form": args.form, "cells": cells, "ordinates": M,
                       "parallelism": f"replicas{ws}", "l2": "inputs larger than L2",
                       "projection_rtol": solver.rtol},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "e2e": e2e,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if ws > 1:
        dist.destroy_process_group()


def measure_e2e(case, steps, ws, form="plain"):
    """Cell-steps/s through the public host-buffer API: every step uploads the
    caller's state (fields, particles, soil) from pinned host memory, advances
    one outer step and downloads the state again; max time over ranks."""
    import torch
    from firewebapp_b200.api import run_3d_spread_gpu_e2e
    res = run_3d_spread_gpu_e2e(case, steps, form=form)
    work, sec = job_totals(res["cells"] * steps, res["seconds"], device="cuda")
    return {"value": work / sec, "unit": UNIT,
            "h2d_bytes_per_step": res["h2d_bytes"] / steps,
            "d2h_bytes_per_step": res["d2h_bytes"] / steps}


if __name__ == "__main__":
    main()
