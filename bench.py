#!/usr/bin/env python
"""Benchmark of the Tier-3 step: 3D solver cell-steps/s on B200.

Workload: the 400 x 120 x 60 cell case (2.88M cells, dx = dy = 0.1 m,
dz = 0.0625 m, DOM S8 with 80 ordinates, U10 = 6 m/s, moisture 0.06,
rho_b = 0.35 kg/m^3, 16 bed particles per surface cell, seeded jitter), plain
FP64 path, projection tolerance 1e-6 (the reference's production default).
Synthetic initial state built from the case deck (no dataset exists for this
solver).  Inputs exceed L2 (state ~0.7 GB, the DOM's octant partial G fields
0.18 GB), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank advances its own
independent replica of the case ("replicas only": the single-case step does
not shard); value = cell-steps/s summed over ranks, time = max over ranks.
``--impl reference`` times the CPU restatement of the reference algorithm
(oracle/) on the host on a bounded slice of the same workload.

At N = 1 the line also carries a ``forms`` block: the mixed-precision and the
learned-preconditioner forms timed the same way on the same case (value, e2e,
CG and DOM iterations per step, fallbacks of the learned solve) and their
ratio to the plain form, and a ``step_roofline``: the per-cell-step
algorithmic bytes of the whole step (distinct fields read and written per
operator, with the measured CG and DOM iteration counts) over the step time.
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
TRAFFIC_PER_CELL = {"dom_sweep": (16.780544e6 + 4.06528e6) / 720000.0}


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
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the mixed and learned forms block of the N = 1 line")
    ap.add_argument("--form", default="plain", choices=["plain", "mixed", "learned"],
                    help="plain: FP64 throughout; mixed: FP32 DOM sweep and multigrid "
                         "preconditioner, pressure tolerance 1e-8; learned: mixed with the "
                         "pressure solve in flexible CG preconditioned by the trained U-Net "
                         "(bf16 tensor-core convolutions), V-cycle fallback on a stall")
    ap.add_argument("--no-clocks", action="store_true",
                    help="skip the clock sampler (diagnostics only; the line then has no clocks)")
    ap.add_argument("--nx", type=int, default=None,
                    help="run the workload cut to its first NX x-cells (profiling)")
    ap.add_argument("--mg-fine-sweeps", type=int, default=None,
                    help="Jacobi sweeps before and after the coarse correction on the finest "
                         "multigrid level (fs_proj_set_fine_sweeps; default: the library's)")
    ap.add_argument("--mg-sweeps", type=int, default=None,
                    help="Jacobi sweeps before and after the coarse correction on every "
                         "multigrid level (fs_proj_configure; with --mg-fine-sweeps the finest "
                         "level keeps its own count; default: the library's)")
    ap.add_argument("--dom-sweep", type=int, default=0,
                    help="force a DOM sweep path (fs_dom_set_sweep_mode); 0 picks automatically")
    ap.add_argument("--dom-kernel", type=int, default=0,
                    help="path 8's sweep kernel (fs_dom_set_sweep_kernel): 0 automatic, "
                         "1 pencil per thread, 2 lane column")
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
    from firewebapp_b200.cases import CFG2
    from firewebapp_b200.solver import Tier3Solver

    case = dict(CFG2, jitter_seed=rank)
    if args.nx:
        from firewebapp_b200.cases import scaled
        case = dict(scaled(CFG2, nx=args.nx), jitter_seed=rank)
    solver = Tier3Solver(case, form=args.form, dom_sweep=args.dom_sweep,
                         mg_sweeps=args.mg_sweeps, mg_fine_sweeps=args.mg_fine_sweeps,
                         dom_kernel=args.dom_kernel)
    cells = solver.n
    M = solver.Omega.shape[0]
    clocks = ClockSampler(local) if not args.no_clocks else None
    tm = time_steps(solver, args.steps, args.warmup, ws, clocks=clocks, kernel_timers=True)
    clk = tm["clocks"] or {"sm_mhz": None, "reasons": ["not sampled"]}
    ms, value, launches, kt = tm["ms"], tm["value"], tm["launches"], tm["kernel_times"]

    # ---- roofline of the dominant bracketed kernel
    peak, peak_src = _peaks()
    roofline = kernel_roofline(solver, kt, args.steps, args.form, peak, peak_src)
    step_roof = step_roofline(solver, tm, peak, peak_src, args.form)

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

    forms = None
    if ws == 1 and not args.nx and args.form == "plain" and not args.no_forms:
        forms = time_forms(case, args, value, e2e)

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
            "roofline": roofline, "step_roofline": step_roof, "cpu_baseline": cpu,
            "clocks": clk, "e2e": e2e, "gpu_launches": launches,
            "iterations_per_step": {"cg": tm["cg_per_step"], "dom_source": tm["dom_per_step"],
                                    "pressure": tm["proj_per_step"]},
            "forms": forms,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if ws > 1:
        dist.destroy_process_group()


def time_steps(solver, steps, warmup, ws, clocks=None, kernel_timers=False):
    """Warm up, then time ``steps`` outer steps with CUDA events on the
    solver's stream (barrier and synchronize on both sides, max over ranks).
    Also counts this library's kernel launches and the CG, pressure and DOM
    source iterations of the timed steps, and the learned solve's fallbacks."""
    import torch
    import torch.distributed as dist
    from firewebapp_b200 import _lib
    lib = _lib.lib()
    for _ in range(warmup):
        solver.step()
    torch.cuda.synchronize()

    def barrier():
        if ws > 1:
            dist.barrier()

    # Objects alive now (torch, numpy, the solver) move to the permanent GC
    # generation, so a full collection during the steps scans only new ones.
    gc.collect()
    gc.freeze()
    if kernel_timers:
        solver.enable_kernel_timers(True)
    fb0 = None
    if solver.form == "learned":
        from firewebapp_b200.learned import fcg_stats
        fb0 = fcg_stats(solver)["fallbacks_total"]
    if clocks:
        clocks.start()
    barrier()
    torch.cuda.synchronize()
    n0 = lib.fs_launch_count()
    cg = proj = dom = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        solver.step()
        d = solver.diag
        cg += sum(d.cg_iters)
        proj += d.proj_iters
        dom += d.dom_iters
    e1.record()
    torch.cuda.synchronize()
    launches = int(lib.fs_launch_count() - n0)
    barrier()
    clk = clocks.stop() if clocks else None
    ms = e0.elapsed_time(e1) / steps
    kt = solver.kernel_times() if kernel_timers else {}
    if kernel_timers:
        solver.enable_kernel_timers(False)
    work, sec = job_totals(solver.n * steps, ms * 1e-3 * steps, device="cuda")
    out = {"ms": 1e3 * sec / steps, "value": work / sec, "launches": launches,
           "kernel_times": kt, "clocks": clk, "cg_per_step": cg / steps,
           "proj_per_step": proj / steps, "dom_per_step": dom / steps}
    if fb0 is not None:
        from firewebapp_b200.learned import fcg_stats
        out["fallbacks"] = fcg_stats(solver)["fallbacks_total"] - fb0
    return out


def kernel_roofline(solver, kt, steps, form, peak, peak_src):
    """Roofline of the dominant bracketed kernel.  Algorithmic bytes per
    launch follow the step's per-operator count (each distinct field read or
    written once per launch, at its storage width).  For the DOM sweep that
    count is the reference's: every one of the M ordinates reads and writes
    its intensity field, plus G read and written, 16 M + 16 bytes per cell
    and source iteration at FP64 (8 M + 8 at FP32); the fused sweep here never
    stores intensities, and its own field traffic (kappa, kappa*B in, eight
    octant partial G fields out) is given beside it."""
    from firewebapp_b200 import _lib
    lib = _lib.lib()
    N = solver.n
    M = solver.Omega.shape[0]
    dom_mode = lib.fs_dom_sweep_mode(solver.dom)
    w = 8.0 if form == "plain" else 4.0
    alg = {
        "dom_sweep": N * (2.0 * w * M + 16.0),
        "species_transport": N * 8.0 * 12,
        "edc": N * 8.0 * 11,
        "turb_diffusion_Y": N * 8.0 * 7,
        "momentum_drag": N * 8.0 * 10,
        "k_epsilon": N * 8.0 * 14,
        "gas_energy_adv": N * 8.0 * 5,
    }
    fused_dom = N * (2.0 * w + 8.0 * w) if dom_mode in (4, 8) else N * (8.0 * M + 16.0)
    dom_k = max((k for k in kt if k in alg), key=lambda k: kt[k][0])
    tot_ms, nl = kt[dom_k]
    avg_ms = tot_ms / max(nl, 1)
    achieved = alg[dom_k] / (avg_ms * 1e-3) / 1e9
    # DRAM bytes per launch of the dominant kernel from an ncu capture of the
    # 100x120x60 slice of this workload (dram__bytes_read.sum + write.sum) with
    # the default sweep (path 8), scaled by the cell count to a full launch
    traffic = (TRAFFIC_PER_CELL.get(dom_k)
               if form == "plain" and (dom_k != "dom_sweep" or dom_mode == 8) else None)
    if traffic is not None:
        traffic *= N
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": traffic, "kernel": dom_k,
           "peak_source": peak_src, "launches": nl, "avg_launch_ms": avg_ms,
           "algorithmic_bytes_per_launch": alg[dom_k], "dom_sweep_path": dom_mode,
           "kernels_ms_per_step": {k: v[0] / steps for k, v in kt.items()}}
    if dom_mode == 8:
        import ctypes
        shape = (ctypes.c_int * 5)()
        if lib.fs_dom_launch_shape(solver.dom, shape) == 0:
            out["dom_cluster"] = dict(zip(("ctas", "rows", "threads", "smem_bytes", "groups"),
                                          list(shape)))
            out["dom_cluster"]["kernel"] = {1: "pencil per thread", 2: "lane column"}.get(
                int(lib.fs_dom_sweep_kernel(solver.dom)), "none")
    if dom_k == "dom_sweep":
        out["fused_sweep_bytes_per_launch"] = fused_dom
        out["fused_sweep_achieved"] = fused_dom / (avg_ms * 1e-3) / 1e9
    return out


def step_roofline(solver, tm, peak, peak_src, form):
    """Whole-step roofline: algorithmic bytes per cell and outer step
    B = B_step + N_SUB B_sub + 128 n_pc f_b + n_cg B_cg + n_src (16 M + 16)
    + 96 (per-operator field counts of the reference loop; n_cg and n_src the
    measured CG and DOM source iterations per step, f_b the bed fraction of
    the cells, n_pc the particles per bed cell), FP64 widths; times cells over
    the step time."""
    g = solver.grid
    M = solver.Omega.shape[0]
    f_b = g.n_z_bed / g.Nz
    n_pc = float(solver.p["n_per_cell"])
    B_step, B_sub, B_cg = 688.0, 328.0 + 24.0 * f_b, 280.0
    n_cg, n_src = tm["cg_per_step"], tm["dom_per_step"]
    terms = {"B_step": B_step, "N_SUB*B_sub": 10 * B_sub, "bed": 128.0 * n_pc * f_b,
             "n_cg*B_cg": n_cg * B_cg, "dom": 96.0 + n_src * (16.0 * M + 16.0)}
    per_cell = sum(terms.values())
    achieved = per_cell * solver.n / (tm["ms"] * 1e-3) / 1e9
    return {"bound": "hbm", "bytes_per_cell_step": per_cell, "terms": terms,
            "bytes_per_step": per_cell * solver.n, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
            "widths": "fp64 field widths for every form"}


def time_forms(case, args, plain_value, plain_e2e):
    """The mixed-precision and learned-preconditioner forms on the same case,
    timed like the headline (device-resident) and end to end."""
    import torch
    from firewebapp_b200.solver import Tier3Solver
    out = {}
    for form in ("mixed", "learned"):
        s = Tier3Solver(case, form=form)
        try:
            tm = time_steps(s, args.steps, args.warmup, 1)
            rec = {"value": tm["value"], "ms_per_step": tm["ms"], "gpu_launches": tm["launches"],
                   "projection_rtol": s.rtol, "cg_per_step": tm["cg_per_step"],
                   "pressure_iterations_per_step": tm["proj_per_step"],
                   "dom_source_per_step": tm["dom_per_step"],
                   "over_plain": tm["value"] / plain_value}
            if "fallbacks" in tm:
                rec["fallbacks"] = tm["fallbacks"]
                rec["pressure_solves"] = int(round(tm["proj_per_step"] * args.steps))
        finally:
            s.close()
            del s
            torch.cuda.empty_cache()
        if not args.no_e2e:
            rec["e2e"] = measure_e2e(case, args.steps, 1, form)
            if plain_e2e:
                rec["e2e_over_plain"] = rec["e2e"]["value"] / plain_e2e["value"]
        out[form] = rec
    out["learned_mixed_over_plain"] = out["learned"]["over_plain"]
    out["mixed_over_plain"] = out["mixed"]["over_plain"]
    return out


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
