"""One outer Tier-3 step in numpy (oracle; test infrastructure).

Restates the production path of the reference loop ``spread_3d.py:1897-3512``
(Lagrangian bed, k-epsilon, EDC, DOM, passive level set) on a state dict
holding the same quantities the reference keeps alive between steps.
"""
from __future__ import annotations

import math

import numpy as np

from . import kernels as K

P0 = 101_325.0
R_AIR = 8.314 / 0.029
G = 9.81
N_SUB = 10


class OracleState:
    """Reference-equivalent state: fields, particles, DOM intensities, clock."""

    def __init__(self, snap, geom, params, Omega, weights, t=0.0, dt_prev=None, step=0):
        self.f = {k: np.array(snap[k], dtype=np.float64) for k in
                  ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s", "alpha_s")}
        self.k_turb = np.array(snap["k_turb"], dtype=np.float64)
        self.eps_turb = np.array(snap["eps_turb"], dtype=np.float64)
        self.nu_t = np.array(snap["nu_t"], dtype=np.float64)
        self.phi = np.array(snap["phi"], dtype=np.float64)
        shp = self.f["rho"].shape
        self.omega = np.array(snap.get("omega", np.zeros(shp)), dtype=np.float64)
        self.q_rad = np.array(snap.get("q_rad", np.zeros(shp)), dtype=np.float64)
        self.q_rad_gas = np.array(snap.get("q_rad_gas", np.zeros(shp)), dtype=np.float64)
        self.T_soil = np.array(snap["T_soil"], dtype=np.float64)
        self.P = {k: np.array(snap["p_" + k]) for k in (
            "x", "y", "z", "alive", "m_solid", "m_water", "m_char", "T_s", "m_water_0", "sav",
            "m_char_max")}
        M = Omega.shape[0]
        self.I_set = (np.array(snap["I_set"], dtype=np.float64) if "I_set" in snap
                      else np.zeros((M,) + shp))
        self.g = geom
        self.p = params
        self.Omega, self.w = Omega, weights
        self.t = float(t)
        self.dt = float(params["dt0"] if dt_prev is None else dt_prev)
        self.step_count = int(step)
        self.lset_step = int(snap.get("lset_step", step))
        self.src = None
        self.M_local = np.zeros(shp)
        self.q_in_soil = np.zeros(shp[1:])
        self.proj_solver = "direct"
        self.proj_rtol = 1.0e-6
        self.precond = None
        self.pressure = (np.array(snap["p_prev"], dtype=np.float64) if "p_prev" in snap
                         else None)

    def snapshot(self):
        out = dict(self.f)
        out.update(k_turb=self.k_turb, eps_turb=self.eps_turb, nu_t=self.nu_t, phi=self.phi,
                   omega=self.omega, q_rad=self.q_rad, q_rad_gas=self.q_rad_gas,
                   T_soil=self.T_soil, I_set=self.I_set)
        for k, v in self.P.items():
            out["p_" + k] = v
        if self.src is not None:
            out["S_pyro_b"] = self.src["S_pyro"]
            out["S_dry_b"] = self.src["S_drying"]
            out["Q_gconv_b"] = self.src["Q_g_conv"]
        return out


def step(S: OracleState):
    """Advance the oracle state by one outer step (spread_3d.py:1897-3512)."""
    g, p, f = S.g, S.p, S.f
    dx, dy, dz, da, db = g["dx"], g["dy"], g["dz"], g["da"], g["db"]
    z_face = g["z_face"]
    nz, ny, nx = f["rho"].shape
    nzb = g["n_z_bed"]
    T_amb = p["T_amb"]
    S.step_count += 1
    # adaptive dt (spread_3d.py:1906-1941)
    u_now = max(float(np.abs(f["u"]).max()), float(np.abs(f["v"]).max()),
                float(np.abs(f["w"]).max()), p["U_mf"], math.sqrt(G * p["h_bed"] * 0.5), 0.1)
    nu_now = max(float(S.nu_t.max()), 1.0e-3)
    dz_min = float(np.min(dz))
    dt_new = min(p["cfl"] * min(dx, dy, dz_min) / u_now, 0.25 * dz_min * dz_min / nu_now, 0.05)
    dt_new = min(dt_new, S.dt * 1.5)
    if dt_new < p["min_dt_s"]:
        dt_new = p["min_dt_s"]
    if not np.isfinite(float(f["T_g"].max())):
        raise RuntimeError("State NaN/Inf")
    S.dt = dt = dt_new
    t = S.t
    ign = t < p["ignition_duration_s"]
    rho_prev = f["rho"].copy()
    f["rho"] = P0 / (R_AIR * np.maximum(f["T_g"], T_amb))
    f["Y_O2"][:, :, 0] = 0.232
    # bed (spread_3d.py:2064-2181)
    Qsx = np.zeros((nz, ny, nx))
    isrc = slice(p["i_src_start"], p["i_src_end"])
    if ign:
        Qsx[:nzb, :, isrc] += 0.80 * (30_000.0 / max(p["h_bed"], 1e-3))
    for kb in range(nzb):
        Qsx[kb] += np.clip(S.q_rad[kb] / dz[kb], -1.0e5, 1.0e5)
    src = K.bed_step(S.P, f["T_g"], f["Y_O2"], Qsx, p["n_per_cell"], dx, dy, dz, z_face,
                     p["h_conv"], p["rho_solid_true"], p["cp_solid"], p["eps_solid"], T_amb,
                     p["view_factor"], p["view_factor_geometric"], p["h_bed"],
                     p["kappa_bed_eff"], dt, p["drying_mode"], p["char_ox_flux_cap"],
                     p["char_ox_ash_exp"])
    S.src = src
    Sp, Sd = src["S_pyro"], src["S_drying"]
    f["T_s"] = K.bed_aggregate(S.P, f["T_s"].shape, dx, dy, z_face, out=f["T_s"], mode=0)
    f["T_s"] = K.bed_hcond(S.P, f["T_s"], f["alpha_s"], dx, dy, z_face, 0.20,
                           p["rho_solid_true"], p["cp_solid"], nzb, dt)
    # drag + momentum
    Fx, Fy, Fz = K.drag_force(f["u"], f["v"], f["w"], f["rho"], f["alpha_s"], p["sav"],
                              p["canopy_C_d"])
    zero2 = np.zeros((nz, ny))
    f["u"], f["v"], f["w"] = K.tentative_velocity(
        f["u"], f["v"], f["w"], f["rho"], f["T_g"], Fx, Fy, Fz, dt, dx, dy, dz, da, db, T_amb,
        g["u_inlet"], zero2, zero2)
    # projection (spread_3d.py:2300-2360)
    drho = (f["rho"] - rho_prev) / dt
    tgt = ((Sp + Sd) - drho) / np.maximum(f["rho"], 0.1)
    n_it = 0
    if S.proj_solver != "direct" and S.precond is None:
        S.precond = K.SeparablePoisson(nz, ny, nx, dx, dy, dz, da, db)
    for _ in range(p["proj_max_iter"]):
        x0 = None if S.pressure is None else S.pressure.reshape(-1)
        f["u"], f["v"], f["w"], pres = K.project(f["u"], f["v"], f["w"], f["rho"], dt, tgt,
                                                 dx, dy, dz, da, db, g["u_inlet"],
                                                 solver=S.proj_solver, rtol=S.proj_rtol,
                                                 x0=x0, precond=S.precond)
        S.pressure = pres
        d = K.divergence(f["u"], f["v"], f["w"], dx, dy, dz, g["u_inlet"]) - tgt
        n_it += 1
        if float(np.max(np.abs(d))) < p["proj_div_tol"]:
            break
    S.pressure = pres
    f["u"] = K.outflow_sponge(f["u"], g["u_inlet"], g["sigma_x"], f["Y_fuel"], 1.0e-3, dt)
    S.k_turb, S.eps_turb, S.nu_t = K.k_epsilon(
        S.k_turb, S.eps_turb, f["u"], f["v"], f["w"], f["T_g"], f["alpha_s"], p["sav"], dt,
        dx, dy, dz, da, db, T_amb, g["u_inlet"], np.full((ny, nx), 1e-8), np.full((ny, nx), 1e-8),
        p["canopy_beta_p"], p["canopy_beta_d"])
    if S.step_count % max(p["dom_subcycle_every"], 1) == 0:
        S.M_local = K.bed_aggregate(S.P, f["T_s"].shape, dx, dy, z_face, mode=1)
        S.q_rad, S.q_rad_gas, S.q_in_soil, _ = K.dom_solve(
            S.I_set, S.Omega, S.w, f["T_s"], f["T_g"], f["alpha_s"], S.omega, p["sav"], T_amb,
            dx, dy, dz, T_soil0=S.T_soil[0], Y_H2O=f["Y_H2O"], rho=f["rho"], M_local=S.M_local)
    S.T_soil = K.soil_step(S.T_soil, S.q_in_soil, dt, g["soil_dz"], g["soil_da"], g["soil_db"],
                           T_amb=T_amb)
    if ign and nzb > 0:
        S.q_rad[nzb - 1, :, isrc] += 240_000.0 * p["ignition_q_mult"]
    n_active = int(K.active_flame(S.omega, f["T_g"], f["Y_fuel"]).sum())
    f["T_g"] = K.gas_energy_adv(f["T_g"], f["u"], f["v"], f["w"], dt, dx, dy, dz, da, db,
                                2.0e-5, T_amb)
    dt_sub = dt / N_SUB
    qdrip_gas = (1.0 - 0.80) * (30_000.0 / max(p["h_bed"], 1e-3))
    for _ in range(N_SUB):
        f["T_g"], f["Y_fuel"], f["Y_O2"], S.omega = K.edc(
            f["rho"], f["T_g"], f["Y_fuel"], f["Y_O2"], S.k_turb, S.eps_turb, f["Y_H2O"],
            0.34, 1100.0, dt_sub, 1, 1.3, 17_000_000.0, p["edc_extinction_enable"])
        St = Sp + Sd
        SF = Sp - f["Y_fuel"] * St
        SO = -f["Y_O2"] * St
        SH = Sd - f["Y_H2O"] * St
        args = (f["rho"], f["u"], f["v"], f["w"])
        f["Y_fuel"] = K.species_transport(f["Y_fuel"], *args, SF, dt_sub, dx, dy, dz, da, db,
                                          1.0e-5, 0.0)
        f["Y_O2"] = K.species_transport(f["Y_O2"], *args, SO, dt_sub, dx, dy, dz, da, db,
                                        1.0e-5, 0.232)
        f["Y_H2O"] = K.species_transport(f["Y_H2O"], *args, SH, dt_sub, dx, dy, dz, da, db,
                                         1.0e-5, 0.0)
        f["Y_O2"] = np.clip(f["Y_O2"], 0.0, 0.232)
        f["Y_H2O"] = np.clip(f["Y_H2O"], 0.0, 1.0)
        for key in ("Y_fuel", "Y_O2", "Y_H2O"):
            f[key] = K.turb_diffusion(f[key], S.nu_t, 0.7, dt_sub, dx, dy, dz, da, db)
        f["Y_O2"] = np.clip(f["Y_O2"], 0.0, 0.232)
        f["Y_fuel"] = np.clip(f["Y_fuel"], 0.0, 1.0)
        f["Y_H2O"] = np.clip(f["Y_H2O"], 0.0, 1.0)
        Qc = np.zeros((nz, ny, nx))
        if ign:
            Qc[:nzb, :, isrc] += qdrip_gas
        Qc += S.q_rad_gas / dz.reshape(-1, 1, 1)
        cp = (1.0 - f["Y_H2O"]) * 1100.0 + f["Y_H2O"] * 2000.0
        deb = (Sp * np.maximum(f["T_g"] - f["T_s"], 0.0)
               + Sd * np.maximum(f["T_g"] - 373.15, 0.0)) * 2000.0
        ginv = dt_sub / (np.maximum(f["rho"], 1.0e-3) * cp)
        f["T_g"] = np.maximum(f["T_g"] + (Qc - src["Q_g_conv"] - deb) * ginv, T_amb)
        f["T_s"] = K.solid_conduction(f["T_s"], f["alpha_s"], dz, da, db, 0.20, 500.0, 1300.0,
                                      dt_sub)
        f["T_g"] = K.turb_diffusion(f["T_g"], S.nu_t, 0.85, dt_sub, dx, dy, dz, da, db)
        f["T_g"] = np.maximum(np.minimum(f["T_g"], 10_000.0), T_amb)
        f["T_s"] = np.maximum(np.minimum(f["T_s"], 10_000.0), T_amb)
    S.lset_step += 1
    if S.lset_step % 10 == 0:
        S.phi = K.levelset_reinit(S.phi, dx, dy, dz)
    f["rho"] = P0 / (R_AIR * np.maximum(f["T_g"], T_amb))
    S.t = t + dt
    S.n_active = n_active
    return dt


def geometry_from_setup(su):
    """Geometry dict for the oracle from a host case set-up."""
    g = su.grid
    return dict(dx=g.dx, dy=g.dy, dz=g.dz_arr, da=g.d_face_above, db=g.d_face_below,
                z_face=g.z_face, n_z_bed=g.n_z_bed, u_inlet=su.u_inlet, sigma_x=su.sigma_sponge,
                soil_dz=su.soil["dz"], soil_da=su.soil["d_above"], soil_db=su.soil["d_below"])
