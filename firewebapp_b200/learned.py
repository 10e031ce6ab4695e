"""The learned form of the pressure solve: a U-Net preconditioner for flexible CG.

No counterpart in the reference (projection_3d.py:756-791 uses BiCGSTAB with
an FFT preconditioner).  The network, its forward and backward kernels and
Adam live in ``csrc/unet.cu``; ``fs_proj_set_learned`` makes
``fs_proj_project`` run flexible CG with z = N(r / rms(r)) and fall back to
the V-cycle PCG from the current iterate when the residual stalls.  The
tolerance is unchanged, so the network's error only costs iterations.

The preconditioner M is a two-level cycle whose coarse correction is the
network: damped-Jacobi pre-smoothing t, r1 = r - S t, s = t + N(r1) (scaled
back to the size of the error), post-smoothing from s.  The sweeps take the
high-frequency error that a bf16 network leaves; the network replaces the
V-cycle's coarse levels.

Training data are the solver's own pressure solves: ``PairLogger`` records,
for every step, the residual r0 at the start of the solve and the correction
e0 = x_solved - x0 that the solve added (S e0 = r0), and turns them into the
network's pair (r1, e1 = e0 - t) with the cycle's own pre-smoothing, both
divided by rms(r1).
"""
from __future__ import annotations

import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr

WEIGHTS = Path(__file__).resolve().parent / "weights" / "unet_precond.npz"

# (cin, cout) of the 11 conv layers, in parameter order (unet.cu kSpec)
CONV_LAYERS = ((16, 16), (16, 16), (16, 32), (32, 32), (32, 48), (48, 48), (48, 64), (64, 64),
               (112, 48), (80, 32), (48, 16))
HEAD_C = 16


def n_params() -> int:
    return sum(27 * ci * co + co for ci, co in CONV_LAYERS) + HEAD_C + 1


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform conv weights (bound sqrt(6 / (27 cin))), zero biases, head
    weights uniform in +-0.25, head bias 0."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co in CONV_LAYERS:
        lim = math.sqrt(6.0 / (27 * ci))
        out.append(rng.uniform(-lim, lim, 27 * ci * co))
        out.append(np.zeros(co))
    out.append(rng.uniform(-0.25, 0.25, HEAD_C))
    out.append(np.zeros(1))
    return np.concatenate(out).astype(np.float32)


class UNetPreconditioner:
    """A U-Net sized for one (nz, ny, nx) grid on the current CUDA device."""

    def __init__(self, nz: int, ny: int, nx: int, params: np.ndarray | None = None,
                 seed: int = 0):
        self.lib = _lib.lib()
        self.shape = (int(nz), int(ny), int(nx))
        self.n = int(nz) * int(ny) * int(nx)
        self.np = int(self.lib.fs_unet_nparams())
        if self.np != n_params():
            raise RuntimeError("parameter layout of the library and the Python side differ")
        h = C.c_void_p()
        check(self.lib.fs_unet_create(int(nz), int(ny), int(nx), C.byref(h)), "fs_unet_create")
        self.h = h
        self.set_params(init_params(seed) if params is None else params)

    @classmethod
    def load(cls, path, nz, ny, nx):
        d = np.load(path)
        net = cls(nz, ny, nx, params=d["params"])
        if "target_scale" in d.files:
            net.set_output_scale(1.0 / float(d["target_scale"]))
        return net

    def set_output_scale(self, c: float):
        """N's output times c is the error estimate (1 / the training target
        scale); c = 0 turns the coarse correction off (smoothing only)."""
        check(self.lib.fs_unet_set_output_scale(self.h, float(c)), "fs_unet_set_output_scale")

    def save(self, path, **meta):
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, params=self.get_params(), **meta)

    def _stream(self):
        return torch.cuda.current_stream().cuda_stream

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.np:
            raise ValueError(f"expected {self.np} parameters, got {p.size}")
        check(self.lib.fs_unet_set_params(self.h, p.ctypes.data, self.np, self._stream()),
              "fs_unet_set_params")

    def get_params(self) -> np.ndarray:
        out = np.empty(self.np, dtype=np.float32)
        check(self.lib.fs_unet_get_params(self.h, out.ctypes.data, self.np, self._stream()),
              "fs_unet_get_params")
        return out

    def get_grads(self) -> np.ndarray:
        out = np.empty(self.np, dtype=np.float32)
        check(self.lib.fs_unet_get_grads(self.h, out.ctypes.data, self.np, self._stream()),
              "fs_unet_get_grads")
        return out

    def _chk(self, t, dtype):
        if t.dtype != dtype or not t.is_cuda or not t.is_contiguous() or t.numel() != self.n:
            raise ValueError(f"expected a contiguous CUDA {dtype} tensor of {self.n} values")

    def apply(self, r: torch.Tensor, z: torch.Tensor):
        """z = N(r / rms(r)) on float64 device tensors."""
        self._chk(r, torch.float64)
        self._chk(z, torch.float64)
        check(self.lib.fs_unet_apply(self.h, ptr(r), ptr(z), self._stream()), "fs_unet_apply")

    def forward(self, r: torch.Tensor) -> torch.Tensor:
        self._chk(r, torch.float32)
        z = torch.empty_like(r)
        check(self.lib.fs_unet_forward(self.h, ptr(r), ptr(z), self._stream()), "fs_unet_forward")
        return z

    def grad(self, r: torch.Tensor, tau: torch.Tensor) -> float:
        self._chk(r, torch.float32)
        self._chk(tau, torch.float32)
        loss = C.c_double()
        check(self.lib.fs_unet_grad(self.h, ptr(r), ptr(tau), C.byref(loss), self._stream()),
              "fs_unet_grad")
        return loss.value

    def train_step(self, r: torch.Tensor, tau: torch.Tensor, lr: float) -> float:
        self._chk(r, torch.float32)
        self._chk(tau, torch.float32)
        loss = C.c_double()
        check(self.lib.fs_unet_train_step(self.h, ptr(r), ptr(tau), float(lr), C.byref(loss),
                                          self._stream()), "fs_unet_train_step")
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.fs_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def attach(solver, net: UNetPreconditioner | None, max_learned: int = 30, stall: float = 0.9):
    """Make ``solver``'s pressure solve use ``net`` (None: the V-cycle again)."""
    if net is not None and net.shape != tuple(solver.shape):
        raise ValueError(f"network grid {net.shape} != solver grid {tuple(solver.shape)}")
    check(solver.lib.fs_proj_set_learned(solver.proj, net.h if net is not None else None,
                                         int(max_learned), float(stall)), "fs_proj_set_learned")


def fcg_stats(solver) -> dict:
    out = (C.c_double * 4)()
    check(solver.lib.fs_proj_fcg_stats(solver.proj, out), "fs_proj_fcg_stats")
    return {"learned_iters": int(out[0]), "vcycle_iters": int(out[1]),
            "fell_back": bool(out[2]), "fallbacks_total": int(out[3])}


class PairLogger:
    """Records (r0, x0) of every pressure solve of ``solver``; ``take`` (after
    a step) returns the network's training pair of the step's last solve:
    (r1, e1) after the learned cycle's pre-smoothing, divided by rms(r1), as
    float32 device tensors.  The solver must be in an FP32 form."""

    def __init__(self, solver):
        self.solver = solver
        f64 = dict(dtype=torch.float64, device=solver.dev)
        self.r0 = torch.zeros(solver.n, **f64)
        self.x0 = torch.zeros(solver.n, **f64)
        check(solver.lib.fs_proj_set_log(solver.proj, ptr(self.r0), ptr(self.x0)),
              "fs_proj_set_log")

    def take(self):
        """(r1_hat, e1_hat) of the last solve, or None when its residual was 0."""
        s = self.solver
        e0 = (s.pressure_view().reshape(-1) - self.x0).contiguous()
        r1 = torch.empty(s.n, dtype=torch.float32, device=s.dev)
        e1 = torch.empty_like(r1)
        check(s.lib.fs_proj_smooth_pair(s.proj, ptr(self.r0), ptr(e0), ptr(r1), ptr(e1),
                                        torch.cuda.current_stream(s.dev).cuda_stream),
              "fs_proj_smooth_pair")
        rms = float(torch.sqrt(torch.mean(r1.double() * r1.double())))
        if not rms > 0.0:
            return None
        return r1 / rms, e1 / rms

    def close(self):
        check(self.solver.lib.fs_proj_set_log(self.solver.proj, None, None), "fs_proj_set_log")


def collect_pairs(cases, steps: int, warmup: int = 5, every: int = 1, device="cuda",
                  on_pair=None):
    """Run every case of ``cases`` (mixed form) for ``warmup + steps`` outer
    steps and return the logged (r_hat, e_hat) pairs of the last ``steps``
    (every ``every``-th step) as float32 device tensors."""
    from .solver import Tier3Solver
    pairs = []
    for case in cases:
        s = Tier3Solver(case, device=device, form="mixed")
        log = PairLogger(s)
        try:
            for k in range(warmup + steps):
                if not s.step():
                    break
                if k >= warmup and (k - warmup) % every == 0:
                    pr = log.take()
                    if pr is not None:
                        pairs.append(pr)
                        if on_pair is not None:
                            on_pair(len(pairs))
        finally:
            log.close()
            s.close()
    return pairs


def train(net: UNetPreconditioner, pairs, iters: int, lr: float = 1e-3, seed: int = 0,
          target_scale: float | None = None, log_every: int = 0):
    """Adam on the mean squared error of N(r_hat) against target_scale * e_hat
    over ``pairs`` (one pair per step, drawn at random; cosine learning rate
    from ``lr`` to lr/20).  ``target_scale`` defaults to 1 / rms of the
    targets, so the targets are O(1).  Returns (losses, target_scale)."""
    if target_scale is None:
        ms = sum(float(torch.mean(e.double() * e.double())) for _, e in pairs) / len(pairs)
        target_scale = 1.0 / math.sqrt(ms) if ms > 0 else 1.0
    rng = np.random.default_rng(seed)
    taus = [(e * target_scale).contiguous() for _, e in pairs]
    losses = []
    for it in range(iters):
        k = int(rng.integers(len(pairs)))
        a = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * it / max(iters, 1))))
        losses.append(net.train_step(pairs[k][0].contiguous(), taus[k], a))
        if log_every and (it + 1) % log_every == 0:
            print(f"train {it + 1}/{iters}: loss {np.mean(losses[-log_every:]):.4e}", flush=True)
    return losses, float(target_scale)


def evaluate(cases, steps: int, weights=WEIGHTS, warmup: int = 3, device="cuda",
             variants=None) -> list[dict]:
    """Held-out comparison at the same tolerance (1e-8): every case stepped
    ``warmup + steps`` times in the mixed form (V-cycle PCG) and in the
    learned form; per case and variant the CG iterations per step (learned
    plus V-cycle after a fallback), the fallback count and the wall time of the
    timed steps.  ``variants``: (name, form, output scale or None,
    learned_max, learned_stall) tuples; the default adds the learned form
    with a looser fallback and the same cycle with the network switched off
    (smoothing only); both stop the learned phase only on a stall (or after
    100 iterations).  A variant that fails (e.g. no convergence within the
    solver's iteration limit) records the error and its completed steps."""
    import time
    from .solver import Tier3Solver
    if variants is None:
        variants = (("vcycle", "mixed", None, 30, 0.9),
                    ("learned", "learned", None, 30, 0.9),
                    ("learned_stall_only", "learned", None, 100, 1.0),
                    ("smoothing_only_stall_only", "learned", 0.0, 100, 1.0))
    out = []
    for ci, case in enumerate(cases):
        for name, form, scale, lmax, stall in variants:
            s = Tier3Solver(case, device=device, form=form, learned_weights=weights,
                            learned_max=lmax, learned_stall=stall)
            try:
                if scale is not None:
                    s.net.set_output_scale(scale)
                for _ in range(warmup):
                    s.step()
                its, lits, fb = [], [], 0
                err = None
                torch.cuda.synchronize(s.dev)
                t0 = time.perf_counter()
                for _ in range(steps):
                    try:
                        if not s.step():
                            break
                    except _lib.FireStepError as e:  # e.g. no convergence in proj_maxiter
                        err = str(e)
                        break
                    its.append(int(sum(s.diag.cg_iters)))
                    if form == "learned":
                        st = fcg_stats(s)
                        lits.append(st["learned_iters"])
                        fb += int(st["fell_back"])
                torch.cuda.synchronize(s.dev)
                wall = time.perf_counter() - t0
            finally:
                s.close()
            out.append({"case": ci, "variant": name, "steps": len(its), "error": err,
                        "cg_iters_mean": float(np.mean(its)), "cg_iters": its,
                        "learned_iters": lits, "fallbacks": fb,
                        "ms_per_step": 1e3 * wall / max(len(its), 1)})
            print(json.dumps(out[-1]), flush=True)
    return out


def time_network(nz: int, ny: int, nx: int, reps: int = 20) -> dict:
    """CUDA-event time of one preconditioner application (fs_unet_apply) and
    one training step on a (nz, ny, nx) grid, after 3 warm-up calls, with the
    network's multiply-add count."""
    net = UNetPreconditioner(nz, ny, nx, seed=1)
    try:
        r = torch.randn(net.n, dtype=torch.float64, device="cuda")
        z = torch.empty_like(r)
        for _ in range(3):
            net.apply(r, z)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            net.apply(r, z)
        e1.record()
        torch.cuda.synchronize()
        apply_ms = e0.elapsed_time(e1) / reps
        r32, tau = r.float(), torch.randn(net.n, device="cuda")
        net.train_step(r32, tau, 1e-6)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(max(reps // 4, 1)):
            net.train_step(r32, tau, 1e-6)
        e1.record()
        torch.cuda.synchronize()
        train_ms = e0.elapsed_time(e1) / max(reps // 4, 1)
    finally:
        net.close()
    dims = [(nz, ny, nx)]
    for _ in range(3):
        dims.append(tuple((v + 1) // 2 for v in dims[-1]))
    level = (0, 0, 1, 1, 2, 2, 3, 3, 2, 1, 0)
    macs = sum(27 * ci * co * math.prod(dims[lv]) for (ci, co), lv in zip(CONV_LAYERS, level))
    return {"grid": [nz, ny, nx], "apply_ms": apply_ms, "train_step_ms": train_ms,
            "conv_gflop": 2e-9 * macs, "apply_tflops": 2e-9 * macs / apply_ms}


def _main(argv=None):
    """python -m firewebapp_b200.learned [train] --cases 4 --steps 60 --iters 1500:
    collects training pairs from seeded cases of the 400x120x60 workload
    (U10 in 2-8 m/s, moisture in 0.02-0.12), trains, writes the weights.
    python -m firewebapp_b200.learned evaluate --seed 200 --cases 5 --steps 20:
    the held-out comparison (``evaluate``) on fresh seeds."""
    import argparse
    import time
    from .cases import learned_cases
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", nargs="?", default="train", choices=["train", "evaluate", "time"])
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--pair-only", action="store_true",
                    help="evaluate: only the V-cycle and the learned form (many seeds)")
    ap.add_argument("--weights", default=None)
    ap.add_argument("--cases", type=int, default=4)
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--every", type=int, default=1)
    ap.add_argument("--iters", type=int, default=1500)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--nx", type=int, default=400)
    ap.add_argument("--out", default=str(WEIGHTS))
    a = ap.parse_args(argv)
    if a.mode == "time":
        print(json.dumps(time_network(60, 120, a.nx, a.reps)))
        return
    cases = learned_cases(a.cases, seed0=a.seed, nx=a.nx)
    if a.mode == "evaluate":
        var = ((("vcycle", "mixed", None, 30, 0.9), ("learned", "learned", None, 30, 0.9))
               if a.pair_only else None)
        evaluate(cases, a.steps, weights=a.weights or str(WEIGHTS), warmup=a.warmup,
                 variants=var)
        return
    t0 = time.time()
    pairs = collect_pairs(cases, a.steps, warmup=a.warmup, every=a.every)
    t1 = time.time()
    print(f"collected {len(pairs)} pairs in {t1 - t0:.1f} s", flush=True)
    net = UNetPreconditioner(60, 120, a.nx, seed=a.seed)
    losses, ts = train(net, pairs, a.iters, lr=a.lr, seed=a.seed, log_every=100)
    t2 = time.time()
    print(f"trained {a.iters} steps in {t2 - t1:.1f} s; loss {np.mean(losses[:50]):.4e} -> "
          f"{np.mean(losses[-50:]):.4e}", flush=True)
    net.save(a.out, target_scale=ts, n_pairs=len(pairs), iters=a.iters, lr=a.lr,
             cases=a.cases, seed=a.seed, steps=a.steps, warmup=a.warmup,
             loss_first=np.mean(losses[:50]), loss_last=np.mean(losses[-50:]))
    print(f"wrote {a.out}")


if __name__ == "__main__":
    _main()
