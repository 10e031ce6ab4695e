"""Per-step diagnostics of a full reference run (64 x 24 x 20 cells, S4,
200 outer steps) for the whole-run comparison of the GPU path.

Runs the reference's own ``run_3d_spread`` through ``refharness`` (one numba
thread, projection rtol 1e-12, the k-epsilon one-sided dT/dz fix, seeded
particle jitter) and records after every step the quantities the comparison
uses: max T_g, max T_s, max omega, max Y_F, the number of cells with
T_s >= T_ign, the peak over x of HRRPUA(x) = (1/Ly) sum_{j,k} omega HOC dz_k dy
and the leading x with T_s >= 600 K.  Writes ``ref_cfg1_run.npz`` next to
this file.

    python tests/golden/make_fullrun.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

HOC_J = 1.7e7
N_STEPS = 200


def main():
    from firewebapp_b200.cases import CFG1
    from firewebapp_b200.grid import build_setup
    from refharness import run_reference
    su = build_setup(CFG1)
    g = su.grid
    dzk = np.asarray(g.dz_arr)[:, None, None]
    T_ign = float(su.params["T_ign"])
    rec = {k: [] for k in ("Tg_max", "Ts_max", "omega_max", "Yf_max", "n_ign", "hrr_peak_x",
                           "lead_x_Ts600")}

    def hook(n, st, cap):
        om = np.asarray(cap["omega"]) if cap.get("omega") is not None else np.zeros_like(st.T_g)
        rec["Tg_max"].append(float(np.max(st.T_g)))
        rec["Ts_max"].append(float(np.max(st.T_s)))
        rec["omega_max"].append(float(np.max(om)))
        rec["Yf_max"].append(float(np.max(st.Y_fuel)))
        rec["n_ign"].append(int(np.sum(st.T_s >= T_ign)))
        hrr = (om * dzk).sum(axis=(0, 1)) * HOC_J * g.dy / g.Ly
        rec["hrr_peak_x"].append(float(hrr.max()))
        hot = np.nonzero((np.asarray(st.T_s) >= 600.0).any(axis=(0, 1)))[0]
        rec["lead_x_Ts600"].append((float(hot.max()) + 0.5) * g.dx if hot.size else np.nan)

    init, snaps, trace = run_reference(CFG1, N_STEPS, capture_steps=[N_STEPS], step_hook=hook)
    out = {k: np.asarray(v) for k, v in rec.items()}
    out["dt"] = np.asarray(trace["dt"][:N_STEPS])
    out["t"] = np.cumsum(out["dt"])
    np.savez_compressed(HERE / "ref_cfg1_run.npz", **out)
    print({k: (v[-1] if v.ndim else v) for k, v in out.items()})


if __name__ == "__main__":
    main()
