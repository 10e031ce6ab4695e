"""The learned form of the pressure solve: a U-Net preconditioner for flexible CG.

No counterpart in the reference (projection_3d.py:756-791 uses BiCGSTAB with
an FFT preconditioner).  The network, its forward and backward kernels and
Adam live in ``csrc/unet.cu``; ``fs_proj_set_learned`` makes
``fs_proj_project`` run flexible CG with z = N(r / rms(r)) and fall back to
the V-cycle PCG from the current iterate when the residual stalls.  The
tolerance is unchanged, so the network's error only costs iterations.

Training data are the solver's own pressure solves: ``PairLogger`` records,
for every step, the residual r0 at the start of the solve and the correction
e = x_solved - x0 that the solve added (S e = r0), both divided by rms(r0).
"""
from __future__ import annotations

import ctypes as C
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
        return cls(nz, ny, nx, params=d["params"])

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
    """Records (r0, e) of every pressure solve of ``solver`` (the last solve of
    a step when ``take`` is called after the step), normalised by rms(r0), as
    float32 device tensors."""

    def __init__(self, solver):
        self.solver = solver
        f64 = dict(dtype=torch.float64, device=solver.dev)
        self.r0 = torch.zeros(solver.n, **f64)
        self.x0 = torch.zeros(solver.n, **f64)
        check(solver.lib.fs_proj_set_log(solver.proj, ptr(self.r0), ptr(self.x0)),
              "fs_proj_set_log")

    def take(self):
        """(r_hat, e_hat) of the last solve, or None when its residual was 0."""
        torch.cuda.synchronize(self.solver.dev)
        rms = float(torch.sqrt(torch.mean(self.r0 * self.r0)))
        if not rms > 0.0:
            return None
        x = self.solver.pressure_view().reshape(-1)
        e = (x - self.x0) / rms
        return (self.r0 / rms).float(), e.float()

    def close(self):
        check(self.solver.lib.fs_proj_set_log(self.solver.proj, None, None), "fs_proj_set_log")


def collect_pairs(cases, steps: int, warmup: int = 5, every: int = 1, device="cuda",
                  on_pair=None):
    """Run every case of ``cases`` (plain form) for ``warmup + steps`` outer
    steps and return the logged (r_hat, e_hat) pairs of the last ``steps``
    (every ``every``-th step) as float32 device tensors."""
    from .solver import Tier3Solver
    pairs = []
    for case in cases:
        s = Tier3Solver(case, device=device, form="plain")
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


def _main(argv=None):
    """python -m firewebapp_b200.learned --cases 4 --steps 60 --iters 1500:
    collects training pairs from seeded cases of the 400x120x60 workload
    (U10 in 2-8 m/s, moisture in 0.02-0.12), trains, writes the weights."""
    import argparse
    import time
    from .cases import learned_cases
    ap = argparse.ArgumentParser()
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
    cases = learned_cases(a.cases, seed0=a.seed, nx=a.nx)
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
