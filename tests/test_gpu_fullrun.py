"""Whole-run comparison with the reference on the 64 x 24 x 20 case (S4, 200
outer steps, 2.8 s of simulated time): the derived quantities (rate of spread
from the leading T_s >= 600 K position, peak HRRPUA, ignited cells, maxima)
must agree within 2 %, and the per-step maxima must track the reference
closely over the first steps.  Reference values: tests/golden/ref_cfg1_run.npz
(tests/golden/make_fullrun.py)."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_cfg1_run.npz"
HOC_J = 1.7e7


def _ros(t, x):
    ok = (t >= 1.0) & np.isfinite(x)
    return np.polyfit(t[ok], x[ok], 1)[0]


def test_full_run_matches_reference():
    import torch
    from firewebapp_b200.cases import CFG1
    from firewebapp_b200.solver import Tier3Solver
    ref = np.load(GOLDEN)
    n = len(ref["dt"])
    s = Tier3Solver(CFG1, projection_cg_rtol=1e-12, proj_maxiter=400)
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
    assert np.allclose(got["t"], ref["t"], rtol=1e-12)
    # first 20 steps: maxima track the reference tightly
    for k in ("Tg_max", "Ts_max", "omega_max", "Yf_max", "hrr_peak_x"):
        np.testing.assert_allclose(got[k][:20], ref[k][:20], rtol=1e-6, atol=1e-12, err_msg=k)
    # whole run: derived quantities within 2 %
    ros_ref, ros_gpu = _ros(ref["t"], ref["lead_x_Ts600"]), _ros(got["t"], got["lead_x_Ts600"])
    assert abs(ros_gpu - ros_ref) <= 0.02 * abs(ros_ref), (ros_gpu, ros_ref)
    for k in ("hrr_peak_x", "Tg_max", "Ts_max"):
        assert abs(got[k].max() - ref[k].max()) <= 0.02 * abs(ref[k].max()), k
    assert abs(got["n_ign"][-1] - ref["n_ign"][-1]) <= 0.02 * ref["n_ign"][-1]
