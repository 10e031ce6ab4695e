"""Per-step diagnostics and snapshot-based ROS of a full reference run
(64 x 24 x 20 cells, S4, 360 outer steps, about 5 s of simulated time) for
the whole-run comparison of the GPU path.

Runs the reference's own ``run_3d_spread`` through ``refharness`` (one numba
thread, projection rtol 1e-12, the k-epsilon one-sided dT/dz fix, seeded
particle jitter) with its snapshot output switched on, and records:

* after every step: max T_g, max T_s, max omega, max Y_F, the number of cells
  with T_s >= T_ign, the peak over x of HRRPUA(x) = (1/Ly) sum_{j,k} omega HOC
  dz_k dy and the leading x with T_s >= 600 K;
* from the reference's own snapshot files (``spread_3d.py:3536-3670``): each
  snapshot's time and leading burned x, read the way the snapshot worker
  reads them (``_cheney_phase16_worker.py:208-231``: float32 T_s >= 600 K in
  any cell of a column, x_mid of the last such column), the worker's ROS_Ts
  fit over them, and the snapshot key set.

Writes ``ref_cfg1_run.npz`` next to this file.

    python tests/golden/make_fullrun.py
"""
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

HOC_J = 1.7e7
N_STEPS = 360
T_IGN_ROS = 600.0


def worker_ros_ts(snap_files):
    """The snapshot worker's ROS_Ts [m/s] and the (t, x) points it fits."""
    ts_t, ts_x = [], []
    for sp in snap_files:
        s = np.load(sp, allow_pickle=True)
        burned = (s["T_s"] >= T_IGN_ROS).any(axis=(0, 1))
        if burned.any():
            ts_t.append(float(s["t"]))
            ts_x.append(float(s["x_mid"][np.where(burned)[0].max()]))
    ros = float("nan")
    if len(ts_t) >= 3:
        late = [i for i, t in enumerate(ts_t) if t >= 1.0]
        if len(late) >= 3:
            ros = float(np.polyfit([ts_t[i] for i in late], [ts_x[i] for i in late], 1)[0])
    return ros, ts_t, ts_x


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

    with tempfile.TemporaryDirectory() as td:
        init, snaps, trace = run_reference(CFG1, N_STEPS, capture_steps=[N_STEPS],
                                           step_hook=hook, snapshot_dir=td)
        files = sorted(Path(td).glob("snap_*.npz"))
        ros_ts, ts_t, ts_x = worker_ros_ts(files)
        snap_t = [float(np.load(f, allow_pickle=True)["t"]) for f in files]
        keys = sorted(np.load(files[0], allow_pickle=True).files)
    out = {k: np.asarray(v) for k, v in rec.items()}
    out["dt"] = np.asarray(trace["dt"][:N_STEPS])
    out["t"] = np.cumsum(out["dt"])
    out["snap_t"] = np.asarray(snap_t)
    out["ros_ts_t"] = np.asarray(ts_t)
    out["ros_ts_x"] = np.asarray(ts_x)
    out["ros_Ts"] = np.float64(ros_ts)
    out["snap_keys"] = np.asarray(keys)
    np.savez_compressed(HERE / "ref_cfg1_run.npz", **out)
    print({k: (v[-1] if v.ndim else v) for k, v in out.items() if k != "snap_keys"})
    print("snapshot keys:", keys)


if __name__ == "__main__":
    main()
