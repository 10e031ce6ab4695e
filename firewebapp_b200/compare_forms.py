"""The mixed-precision form against the plain FP64 form on the same seeded cases.

For each case (by default the 400x120x60 workload with U10 ~ U(2, 8) m/s and
moisture ~ U(0.02, 0.12) from a seeded PCG64 stream, ``cases.learned_cases``):

* per-field error: both forms stepped side by side from the same initial
  state; relative L2 of every state field after the requested steps (the
  velocity components against the norm of the whole velocity vector, since a
  crosswind component can be orders of magnitude smaller than the others);
* derived quantities: a run of each form to ``t_end`` simulated seconds
  through ``api.run_3d_spread_gpu``; ROS_Ts the way the reference's snapshot
  worker computes it (``api.ros_from_snapshots``) and the peak HRRPUA, with
  their relative differences.

Usage::

    python -m firewebapp_b200.compare_forms --cases 3 --seed0 300 --steps 10 50 --t-end 6

prints one JSON line per case and a summary table.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

FIELDS = ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s", "k_turb", "eps_turb",
          "nu_t", "omega", "q_rad", "q_rad_gas", "T_soil", "p_T_s", "p_m_solid", "p_m_water")
VEL = ("u", "v", "w")


def field_errors(plain: dict, mixed: dict) -> dict:
    """Relative L2 of every field of ``mixed`` against ``plain`` (velocity
    components against the norm of the plain velocity vector)."""
    out = {}
    vnorm = math.sqrt(sum(float(np.linalg.norm(plain[k])) ** 2 for k in VEL))
    for k in FIELDS:
        a = np.asarray(plain[k], dtype=np.float64).ravel()
        b = np.asarray(mixed[k], dtype=np.float64).ravel()
        den = vnorm if k in VEL else float(np.linalg.norm(a))
        out[k] = float(np.linalg.norm(b - a) / den) if den > 0 else float(np.linalg.norm(b - a))
    return out


def compare_steps(case: dict, steps=(10,), device="cuda") -> dict:
    """Per-field errors of the mixed form after each count in ``steps``."""
    from .solver import Tier3Solver
    a = Tier3Solver(case, device=device, form="plain")
    b = Tier3Solver(case, device=device, form="mixed")
    out = {}
    try:
        n = 0
        for target in sorted(steps):
            while n < target:
                ra, rb = a.step(), b.step()
                n += 1
                if not (ra and rb):
                    break
            out[n] = field_errors(a.state(), b.state())
            if n < target:
                break
    finally:
        a.close()
        b.close()
    return out


def compare_run(case: dict, t_end: float, device="cuda") -> dict:
    """ROS_Ts and peak HRRPUA of both forms over a run to ``t_end`` seconds."""
    from .api import run_3d_spread_gpu
    res = {}
    for form in ("plain", "mixed"):
        r = run_3d_spread_gpu(case, t_end=t_end, device=device, form=form)
        res[form] = {"ros_Ts": r.ros_Ts, "hrrpua_peak": r.hrrpua_peak,
                     "snapshots": len(r.snap_t), "n_cells_ignited": r.n_cells_ignited}

    def rel(key):
        p, m = res["plain"][key], res["mixed"][key]
        if not (np.isfinite(p) and np.isfinite(m)) or p == 0:
            return float("nan")
        return float(abs(m - p) / abs(p))
    res["ros_rel_diff"] = rel("ros_Ts")
    res["hrrpua_rel_diff"] = rel("hrrpua_peak")
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--cases", type=int, default=3)
    ap.add_argument("--seed0", type=int, default=300)
    ap.add_argument("--nx", type=int, default=400)
    ap.add_argument("--steps", type=int, nargs="+", default=[10, 50])
    ap.add_argument("--t-end", type=float, default=6.0,
                    help="simulated seconds of the ROS runs (0: skip them)")
    args = ap.parse_args(argv)
    from .cases import learned_cases
    rows = []
    for k, case in enumerate(learned_cases(args.cases, seed0=args.seed0, nx=args.nx)):
        rec = {"seed": args.seed0 + k, "U10": case["wind_speed_m_s"],
               "moisture": case["initial_moisture_frac"]}
        rec["errors"] = {str(n): e for n, e in compare_steps(case, args.steps).items()}
        if args.t_end > 0:
            rec["run"] = compare_run(case, args.t_end)
        print(json.dumps(rec), flush=True)
        rows.append(rec)
    # summary: worst field error per step count, ROS/HRRPUA differences
    for n in sorted({int(s) for r in rows for s in r["errors"]}):
        worst = {}
        for r in rows:
            for f, v in r["errors"].get(str(n), {}).items():
                worst[f] = max(worst.get(f, 0.0), v)
        print(f"after {n} steps, max over cases: " +
              ", ".join(f"{f} {v:.1e}" for f, v in worst.items()))
    for r in rows:
        if "run" in r:
            p, m = r["run"]["plain"], r["run"]["mixed"]
            print(f"seed {r['seed']} U10 {r['U10']:.2f} moisture {r['moisture']:.3f}: ROS_Ts "
                  f"{p['ros_Ts']:.4f} / {m['ros_Ts']:.4f} m/s (diff {r['run']['ros_rel_diff']:.2%}), "
                  f"peak HRRPUA {p['hrrpua_peak']:.4g} / {m['hrrpua_peak']:.4g} "
                  f"(diff {r['run']['hrrpua_rel_diff']:.2%})")


if __name__ == "__main__":
    main()
