"""Whole-run comparison with the reference on the 64 x 24 x 20 case (S4, 360
outer steps, about 5 s of simulated time).  Reference values:
tests/golden/ref_cfg1_run.npz (tests/golden/make_fullrun.py, the reference's
own run with its snapshot output switched on).

* Per-step maxima, ignited cells and peak HRRPUA from ``Tier3Solver`` at the
  parity tolerance (projection rtol 1e-12) and at the production tolerance
  (the plain form's 1e-6): derived quantities within 2 %.
* The driver-level drop-in ``run_3d_spread_gpu`` with snapshots: its files
  carry the reference's snapshot keys at the reference's snapshot instants,
  and ROS_Ts, computed the way the snapshot worker computes it
  (``_cheney_phase16_worker.py:208-231``) both by the product
  (``api.ros_from_snapshots``) and from the written files, is within 2 % of
  the reference run's, for the plain and the mixed-precision forms.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_cfg1_run.npz"
HOC_J = 1.7e7


def _ros(t, x):
    ok = (t >= 1.0) & np.isfinite(x)
    return np.polyfit(t[ok], x[ok], 1)[0]


@pytest.mark.parametrize("rtol", [1e-12, None])
def test_full_run_matches_reference(rtol):
    import torch
    from firewebapp_b200.cases import CFG1
    from firewebapp_b200.solver import Tier3Solver
    ref = np.load(GOLDEN)
    n = len(ref["dt"])
    s = Tier3Solver(CFG1, projection_cg_rtol=rtol, proj_maxiter=400)
    g = s.grid
    dzk = s.dz_t.view(-1, 1, 1)
    T_ign = float(s.p["T_ign"])
    rec = {k: [] for k in ("Tg_max", "Ts_max", "omega_max", "Yf_max", "n_ign", "hrr_peak_x",
                           "lead_x_Ts600", "t")}
    for _ in range(n):
        assert s.step()
        f, w = s.f, s.w
        rec["Tg_max"].append(float(f["T_g"].max()))
        rec["Ts_max"].append(float(f["T_s"].max()))
        rec["omega_max"].append(float(w["omega"].max()))
        rec["Yf_max"].append(float(f["Y_fuel"].max()))
        rec["n_ign"].append(int((f["T_s"] >= T_ign).sum()))
        hrr = (w["omega"] * dzk).sum(dim=(0, 1)) * HOC_J * g.dy / g.Ly
        rec["hrr_peak_x"].append(float(hrr.max()))
        hot = torch.nonzero((f["T_s"] >= 600.0).any(dim=0).any(dim=0))
        rec["lead_x_Ts600"].append((float(hot.max()) + 0.5) * g.dx if hot.numel() else np.nan)
        rec["t"].append(s.t)
    s.close()
    got = {k: np.asarray(v) for k, v in rec.items()}
    if rtol is not None:
        assert np.allclose(got["t"], ref["t"], rtol=1e-12)
        # first 20 steps: maxima track the reference tightly
        for k in ("Tg_max", "Ts_max", "omega_max", "Yf_max", "hrr_peak_x"):
            np.testing.assert_allclose(got[k][:20], ref[k][:20], rtol=1e-6, atol=1e-12,
                                       err_msg=k)
    else:
        assert np.allclose(got["t"], ref["t"], rtol=1e-3)
    # whole run: derived quantities within 2 %
    ros_ref, ros_gpu = _ros(ref["t"], ref["lead_x_Ts600"]), _ros(got["t"], got["lead_x_Ts600"])
    assert abs(ros_gpu - ros_ref) <= 0.02 * abs(ros_ref), (ros_gpu, ros_ref)
    for k in ("hrr_peak_x", "Tg_max", "Ts_max"):
        assert abs(got[k].max() - ref[k].max()) <= 0.02 * abs(ref[k].max()), k
    assert abs(got["n_ign"][-1] - ref["n_ign"][-1]) <= 0.02 * ref["n_ign"][-1]


def _worker_ros_from_files(files):
    """ROS_Ts from snapshot files, read as the snapshot worker reads them."""
    ts_t, ts_x = [], []
    for sp in files:
        s = np.load(sp, allow_pickle=True)
        burned = (s["T_s"] >= 600.0).any(axis=(0, 1))
        if burned.any():
            ts_t.append(float(s["t"]))
            ts_x.append(float(s["x_mid"][np.where(burned)[0].max()]))
    late = [i for i, t in enumerate(ts_t) if t >= 1.0]
    assert len(ts_t) >= 3 and len(late) >= 3
    return float(np.polyfit([ts_t[i] for i in late], [ts_x[i] for i in late], 1)[0])


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_driver_snapshots_and_ros_match_reference(tmp_path, form):
    from firewebapp_b200.api import run_3d_spread_gpu
    from firewebapp_b200.cases import CFG1
    ref = np.load(GOLDEN)
    n = len(ref["dt"])
    res = run_3d_spread_gpu(CFG1, n_steps=n, snapshot_dir=tmp_path, form=form)
    files = sorted(tmp_path.glob("snap_*.npz"))
    # the reference writes a snapshot after step 1 and then every 1 s of
    # simulated time; its run stops inside step n, before that step's snapshot
    ref_t = ref["snap_t"]
    assert len(files) >= len(ref_t)
    got_t = np.array([float(np.load(f, allow_pickle=True)["t"]) for f in files])
    np.testing.assert_allclose(got_t[:len(ref_t)], ref_t, rtol=1e-3)
    assert sorted(np.load(files[0], allow_pickle=True).files) == sorted(ref["snap_keys"].tolist())
    # the product's ROS_Ts equals the worker's formula applied to its own files
    ros_files = _worker_ros_from_files(files)
    assert abs(res.ros_Ts - ros_files) <= 1e-9 * abs(ros_files), (res.ros_Ts, ros_files)
    ros_ref = float(ref["ros_Ts"])
    assert np.isfinite(ros_ref) and ros_ref > 0.0
    assert abs(res.ros_Ts - ros_ref) <= 0.02 * ros_ref, (res.ros_Ts, ros_ref)
    # per-step diagnostics as the reference appends them (spread_3d.py:3503-3512)
    assert len(res.diag_t) == n and len(res.diag_n_ign) == n
    assert all(isinstance(v, int) for v in res.diag_proj_n_iter)
    np.testing.assert_allclose(np.max(res.diag_Tg_max), np.max(ref["Tg_max"]), rtol=0.02)
    np.testing.assert_allclose(res.hrrpua_peak, np.max(ref["hrr_peak_x"]), rtol=0.02)
    assert abs(res.diag_n_ign[-1] - ref["n_ign"][-1]) <= 0.02 * ref["n_ign"][-1]
